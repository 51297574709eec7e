"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/_ref/libref_ingest.so: the reference's own scene loader
(SceneLoader::LoadSceneFromXML with MaterialUtils, the vendored tinyxml2 and tinyobjloader)
compiled here from its sources by `make -C oracle ref`. load_xml() returns what the reference's
loader put into its Scene, in the same form as nomad_b200.LoadedScene, so the two can be compared
array by array. Texture images are not decoded on either side (every texture index is -1).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_ingest.so")
_lib = None
_P = C.c_void_p


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle ref` where the reference exists")
        lib = C.CDLL(LIB_PATH)
        lib.ref_load_xml.argtypes = [C.c_char_p, C.POINTER(_P)]
        lib.ref_load_xml.restype = C.c_int
        lib.ref_loaded_counts.argtypes = [_P, C.POINTER(C.c_uint32)]
        lib.ref_loaded_counts.restype = None
        lib.ref_loaded_arrays.argtypes = [_P] + [_P] * 9 + [C.c_char_p, C.c_uint32]
        lib.ref_loaded_arrays.restype = None
        lib.ref_loaded_free.argtypes = [_P]
        lib.ref_loaded_free.restype = None
        _lib = lib
    return _lib


def load_xml(path: str):
    """The reference loader's result for `path`, or None when it reports failure."""
    from nomad_b200.native import CameraKeyframe, ObserverCamera, SceneSettings

    lib = load()
    h = _P()
    if lib.ref_load_xml(os.fsencode(path), C.byref(h)) != 0:
        return None
    try:
        cnt = (C.c_uint32 * 4)()
        lib.ref_loaded_counts(h, cnt)
        n, m, k, has_obs = (int(x) for x in cnt)
        out = {"prim_type": np.zeros(n, np.int32), "prim_geom": np.zeros((n, 15), np.float32),
               "prim_material": np.zeros((n, 20), np.float32), "object_first": np.zeros(m, np.uint32),
               "object_prims": np.zeros(m, np.uint32), "object_mesh_group": np.zeros(m, np.int32)}
        settings = SceneSettings()
        keys = (CameraKeyframe * max(k, 1))()
        obs = ObserverCamera()
        env = C.create_string_buffer(4096)
        lib.ref_loaded_arrays(h, *(out[x].ctypes.data for x in ("prim_type", "prim_geom", "prim_material",
                                                                  "object_first", "object_prims",
                                                                  "object_mesh_group")),
                              C.addressof(settings), C.addressof(keys), C.addressof(obs), env, 4096)
    finally:
        lib.ref_loaded_free(h)
    out["settings"] = settings.as_dict()
    out["keyframes"] = [
        {"frame": x.frame, "position": tuple(x.position), "look_at": tuple(x.look_at), "up": tuple(x.up),
         "aperture": x.aperture, "focus_distance": x.focus_distance} for x in list(keys)[:k]]
    out["observer"] = ({"position": tuple(obs.position), "look_at": tuple(obs.look_at), "up": tuple(obs.up),
                        "vertical_fov": obs.vertical_fov, "aperture": obs.aperture,
                        "focus_distance": obs.focus_distance} if has_obs else None)
    out["environment_texture"] = env.value.decode()
    return out
