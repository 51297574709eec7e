"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/_ref/libref_nomad.so: the reference's own code compiled here from
its sources (SceneBVH.cpp + Scene.cpp for the builder; Shaders/PathTracing.h for the
traversal, through a Metal-compatibility header). Built by `make -C oracle ref` only where the
reference sources are present; the .so travels with the repository snapshot. When it is
absent, available() is False and callers use the scalar port (oracle.py).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_nomad.so")
_lib = None
_P = C.c_void_p
HIT_DTYPE = np.dtype([("inst", "<i4"), ("prim", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle ref` where the reference exists")
        lib = C.CDLL(LIB_PATH)
        lib.ref_build_scene.argtypes = [C.c_uint32, _P, _P, _P, C.c_uint32, _P, _P, C.POINTER(_P)]
        lib.ref_build_scene.restype = C.c_int
        lib.ref_scene_counts.argtypes = [_P, C.POINTER(C.c_uint32)]
        lib.ref_scene_counts.restype = None
        lib.ref_scene_arrays.argtypes = [_P, _P, _P, _P, _P, _P, _P]
        lib.ref_scene_arrays.restype = None
        lib.ref_scene_free.argtypes = [_P]
        lib.ref_scene_free.restype = None
        lib.ref_trace.argtypes = [_P, _P, C.c_uint32, _P, _P, _P, _P, _P, C.c_uint32, _P,
                                  C.c_uint64, _P, _P, C.c_uint32, C.c_int]
        lib.ref_trace.restype = C.c_int
        _lib = lib
    return _lib


def _p(a):
    return a.ctypes.data


def build_scene(scene):
    """Runs the reference's Scene::addObject + Scene::buildBVH + create*Buffer on a HostScene;
    returns a dict of the packed arrays (same layout as nomad_b200.SceneBVH)."""
    lib = load()
    h = _P()
    rc = lib.ref_build_scene(scene.prim_count, _p(scene.prim_type), _p(scene.prim_geom),
                             _p(scene.prim_material), scene.object_count, _p(scene.object_first),
                             _p(scene.object_prims), C.byref(h))
    assert rc == 0, rc
    try:
        cnt = (C.c_uint32 * 4)()
        lib.ref_scene_counts(h, cnt)
        nb_, nt, n_prim, n_obj = cnt
        out = {"bvh_nodes": np.zeros(nb_ * 8, np.float32), "tlas_nodes": np.zeros(nt * 8, np.float32),
               "prims": np.zeros(n_prim * 28, np.float32), "materials": np.zeros(n_prim * 20, np.float32),
               "prim_indices": np.zeros(n_prim, np.int32), "blas_root": np.zeros(n_obj, np.int32)}
        lib.ref_scene_arrays(h, _p(out["bvh_nodes"]), _p(out["tlas_nodes"]), _p(out["prims"]),
                             _p(out["materials"]), _p(out["prim_indices"]), _p(out["blas_root"]))
        return out
    finally:
        lib.ref_scene_free(h)


def closest(sb, rays, threads=0, active=None, blas_root=None, stats=None):
    """The reference's firstHitTLAS (PathTracing.h:961-1066), run verbatim on the CPU, over the
    SceneBVH arrays of `sb`. stats, when given, is the reference's primitiveRayStats buffer
    (2 * prim_count + 2 uint32) and receives its atomic leaf-test counts."""
    lib = load()
    rays = np.ascontiguousarray(rays)
    active = np.ones(sb.prim_count, np.uint8) if active is None else np.ascontiguousarray(active, np.uint8)
    root = (np.ascontiguousarray(sb.instances["blas_root_index"], np.int32) if blas_root is None
            else np.ascontiguousarray(blas_root, np.int32))
    out = np.empty(rays.shape[0], HIT_DTYPE)
    st = _p(stats) if stats is not None else None
    rc = lib.ref_trace(_p(sb.bvh_nodes), _p(sb.tlas_nodes), sb.tlas_nodes.size // 8, _p(sb.prims),
                       _p(np.ascontiguousarray(sb.prim_indices, np.int32)), _p(active), _p(root),
                       _p(np.ascontiguousarray(sb.prim_object, np.int32)), sb.prim_count,
                       _p(rays), rays.shape[0], _p(out), st, threads, 0)
    assert rc == 0, rc
    return out
