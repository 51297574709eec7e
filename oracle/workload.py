"""ORACLE — test infrastructure only: the bench's reference arm's workload.

The reference arm times the reference's own traversal (oracle/reference.py, firstHitTLAS compiled
from PathTracing.h) and must map nothing of this repository's library. This module builds the
same workload without it: the seeded city from the generator's source compiled on its own
(oracle/_build/libsynth.so, from nomad_b200/csrc/host/synth.cpp), the SceneBVH arrays from the
reference's own builder (Scene::buildBVH, SceneBVH.cpp, through oracle/reference.py), the primary
rays and the bounce rays from the numpy ray helpers (nomad_b200/rays.py, which loads no library),
and the primary hits that seed the bounces from the reference's own traversal.
"""
from __future__ import annotations

import ctypes as C
import os
import types

import numpy as np

from . import reference as ref

_HERE = os.path.dirname(os.path.abspath(__file__))
SYNTH_PATH = os.path.join(_HERE, "_build", "libsynth.so")
_lib = None
_P = C.c_void_p


class _Desc(C.Structure):  # nomad_scene_desc (include/nomad_scene.h)
    _fields_ = [("prim_count", C.c_uint32), ("prim_type", C.POINTER(C.c_int32)),
                ("prim_geom", C.POINTER(C.c_float)), ("prim_material", C.POINTER(C.c_float)),
                ("object_count", C.c_uint32), ("object_first", C.POINTER(C.c_uint32)),
                ("object_prims", C.POINTER(C.c_uint32))]


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(SYNTH_PATH):
            raise RuntimeError(f"{SYNTH_PATH} missing: run `make -C oracle`")
        lib = C.CDLL(SYNTH_PATH)
        lib.nomad_synth_city.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32,
                                         C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(_P)]
        lib.nomad_synth_city.restype = C.c_int32
        lib.nomad_scene_owned_desc.argtypes = [_P, C.POINTER(_Desc)]
        lib.nomad_scene_owned_desc.restype = C.c_int32
        lib.nomad_scene_owned_free.argtypes = [_P]
        lib.nomad_scene_owned_free.restype = None
        _lib = lib
    return _lib


def synth_city(seed, grid=32, size_m=1000.0, target_tris=2_500_000, median_tris=1000, max_tris=200_000,
               emissive_quads=64, emissive_tris=0, emissive_sigma=1.5, grid_z=0):
    """nomad_synth_city (same arguments as nomad_b200.synth_city) as a namespace of arrays."""
    lib = _load()
    h = _P()
    rc = lib.nomad_synth_city(seed, grid, grid_z or grid, size_m, target_tris, median_tris, max_tris,
                              emissive_quads, emissive_tris, emissive_sigma, C.byref(h))
    assert rc == 0, rc
    try:
        d = _Desc()
        assert lib.nomad_scene_owned_desc(h, C.byref(d)) == 0
        n, m = d.prim_count, d.object_count
        return types.SimpleNamespace(
            prim_count=n, object_count=m,
            prim_type=np.ctypeslib.as_array(d.prim_type, (n,)).copy(),
            prim_geom=np.ctypeslib.as_array(d.prim_geom, (n * 15,)).copy().reshape(-1, 15),
            prim_material=np.ctypeslib.as_array(d.prim_material, (n * 20,)).copy().reshape(-1, 20),
            object_first=np.ctypeslib.as_array(d.object_first, (m,)).copy(),
            object_prims=np.ctypeslib.as_array(d.object_prims, (m,)).copy())
    finally:
        lib.nomad_scene_owned_free(h)


def scene_bvh(scene):
    """The SceneBVH arrays of `scene` from the reference's own builder, in the attribute layout
    reference.closest reads (the same as nomad_b200.SceneBVH's)."""
    r = ref.build_scene(scene)
    inst = np.zeros(scene.object_count, np.dtype([("blas_root_index", "<i4"), ("prim_base", "<u4"),
                                                  ("prim_count", "<u4"), ("prim_index_base", "<u4")]))
    inst["blas_root_index"] = r["blas_root"]
    return types.SimpleNamespace(
        bvh_nodes=r["bvh_nodes"], tlas_nodes=r["tlas_nodes"], prims=r["prims"], materials=r["materials"],
        prim_indices=r["prim_indices"], instances=inst, prim_count=scene.prim_count,
        object_count=scene.object_count,
        prim_object=np.repeat(np.arange(scene.object_count, dtype=np.int32), scene.object_prims.astype(np.int64)))


def city_rays(sb, camera, spp, seed, bounce_seed, sample=None, threads=0):
    """Primary rays of `camera` (spp jittered per pixel), optionally a random sample of them,
    followed by one diffuse bounce per primary hit, the hits from the reference's traversal."""
    from nomad_b200.rays import bounce_rays  # numpy only

    primary = camera.primary_rays(spp, seed=seed)
    if sample is not None:
        primary = primary[np.random.default_rng(7).permutation(primary.shape[0])[:sample]]
    hits = ref.closest(sb, primary, threads=threads)
    return np.concatenate([primary, bounce_rays(primary, hits, sb.prims, seed=bounce_seed)])
