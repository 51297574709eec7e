"""ORACLE — test infrastructure only (the checker, never the product).

ctypes wrapper of oracle/_build/liboracle.so, the scalar C++ restatement of the reference's
traversal (see contract.cpp for the file:line map). Only tests/, __graft_entry__.smoke() and
bench.py's CPU legs import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libref_nomad.so")

HIT_DTYPE = np.dtype([("inst", "<i4"), ("prim", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
MODE_REFERENCE_ORDER, MODE_NEAR_FIRST, MODE_BRUTE = 0, 1, 2

_lib = None
_P = C.c_void_p


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        lib = C.CDLL(LIB_PATH)
        common = [_P, _P, C.c_uint32, _P, _P, _P, _P, _P, C.c_uint32, _P, C.c_uint64]
        lib.oracle_trace_closest.argtypes = common + [_P, C.c_int, C.c_uint32]
        lib.oracle_trace_closest.restype = C.c_int
        lib.oracle_trace_any.argtypes = common + [_P, C.c_int, C.c_uint32]
        lib.oracle_trace_any.restype = C.c_int
        lib.oracle_trace_work.argtypes = common + [_P, _P, C.c_uint32]
        lib.oracle_trace_work.restype = C.c_int
        _lib = lib
    return _lib


def _p(a):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


class OracleScene:
    """The SceneBVH arrays plus residency state the oracle traverses."""

    def __init__(self, sb, active=None, blas_root=None):
        self.bvh = np.ascontiguousarray(sb.bvh_nodes, np.float32)
        self.tlas = np.ascontiguousarray(sb.tlas_nodes, np.float32)
        self.prims = np.ascontiguousarray(sb.prims, np.float32)
        self.prim_indices = np.ascontiguousarray(sb.prim_indices, np.int32)
        self.prim_object = np.ascontiguousarray(sb.prim_object, np.int32)
        self.object_count = int(sb.object_count)
        self.active = (np.ones(sb.prim_count, np.uint8) if active is None
                       else np.ascontiguousarray(active, np.uint8))
        self.blas_root = (np.ascontiguousarray(sb.instances["blas_root_index"], np.int32)
                          if blas_root is None else np.ascontiguousarray(blas_root, np.int32))

    def _args(self, rays):
        rays = np.ascontiguousarray(rays)
        assert rays.dtype.itemsize == 32
        return (_p(self.bvh), _p(self.tlas), self.tlas.size // 8, _p(self.prims),
                _p(self.prim_indices), _p(self.active), _p(self.blas_root), _p(self.prim_object),
                self.object_count, _p(rays), rays.shape[0]), rays

    def closest(self, rays, mode=MODE_REFERENCE_ORDER, threads=0):
        args, rays = self._args(rays)
        out = np.empty(rays.shape[0], HIT_DTYPE)
        assert load().oracle_trace_closest(*args, _p(out), mode, threads) == 0
        return out

    def any(self, rays, mode=MODE_REFERENCE_ORDER, threads=0):
        args, rays = self._args(rays)
        out = np.empty(rays.shape[0], np.uint8)
        assert load().oracle_trace_any(*args, _p(out), mode, threads) == 0
        return out

    def work(self, rays, threads=0):
        args, rays = self._args(rays)
        out = np.empty((rays.shape[0], 4), np.uint32)
        hits = np.empty(rays.shape[0], HIT_DTYPE)
        assert load().oracle_trace_work(*args, _p(out), _p(hits), threads) == 0
        return out, hits


def algorithmic_bytes(work: np.ndarray) -> np.ndarray:
    """Bytes per ray: 32 per box tested, 48+4 per primitive test (positions + index),
    16 per instance record, 48 per closest hit (the hit's frame float4 4..6)."""
    w = work.astype(np.int64)
    return 32 * w[:, 0] + 52 * w[:, 1] + 16 * w[:, 2] + 48 * w[:, 3]


def render(os_: "OracleScene", materials, views, pixels=None, obj_hits=False, threads=0):
    """Scalar path tracer (pathtrace.cpp) on the listed global pixel indices of the views
    (all pixels when None). Returns (rgb[n,3], obj_hits or None, stats[4])."""
    lib = load()
    if not hasattr(lib, "_render_bound"):
        lib.oracle_render.argtypes = [_P, _P, C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_uint32,
                                      C.c_uint32, _P, C.c_uint32, _P, C.c_uint64, _P, _P, _P,
                                      C.c_uint32]
        lib.oracle_render.restype = C.c_int
        lib._render_bound = True
    views = np.ascontiguousarray(views).reshape(-1)
    if pixels is None:
        total = int((views["width"].astype(np.int64) * views["height"]).sum())
        pixels = np.arange(total, dtype=np.uint64)
    pixels = np.ascontiguousarray(pixels, np.uint64)
    mats = np.ascontiguousarray(materials, np.float32)
    out = np.zeros((pixels.size, 3), np.float32)
    hits = np.zeros(os_.object_count, np.uint32) if obj_hits else None
    stats = np.zeros(4, np.uint64)
    rc = lib.oracle_render(_p(os_.bvh), _p(os_.tlas), os_.tlas.size // 8, _p(os_.prims), _p(mats),
                           _p(os_.prim_indices), _p(os_.active), _p(os_.blas_root),
                           _p(os_.prim_object), os_.object_count, os_.prims.size // 28,
                           _p(views), views.shape[0], _p(pixels), pixels.size, _p(out),
                           _p(hits) if hits is not None else None, _p(stats), threads)
    assert rc == 0
    return out, hits, stats


def render_tape(os_: "OracleScene", materials, views, tapes, pixels=None, threads=0):
    """render() in tape mode: tapes[q] (float32, T per listed pixel) are the pixel's random numbers,
    drawn in the reference's order (pathtrace.cpp, Draws). Returns rgb[n, 3]."""
    lib = load()
    if not hasattr(lib, "_render_tape_bound"):
        lib.oracle_render_tape.argtypes = [_P, _P, C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_uint32, C.c_uint32,
                                           _P, C.c_uint32, _P, C.c_uint64, _P, C.c_uint32, _P, C.c_uint32]
        lib.oracle_render_tape.restype = C.c_int
        lib._render_tape_bound = True
    views = np.ascontiguousarray(views).reshape(-1)
    if pixels is None:
        total = int((views["width"].astype(np.int64) * views["height"]).sum())
        pixels = np.arange(total, dtype=np.uint64)
    pixels = np.ascontiguousarray(pixels, np.uint64)
    tapes = np.ascontiguousarray(tapes, np.float32)
    assert tapes.shape[0] == pixels.size
    out = np.zeros((pixels.size, 3), np.float32)
    rc = lib.oracle_render_tape(_p(os_.bvh), _p(os_.tlas), os_.tlas.size // 8, _p(os_.prims),
                                _p(np.ascontiguousarray(materials, np.float32)), _p(os_.prim_indices),
                                _p(os_.active), _p(os_.blas_root), _p(os_.prim_object), os_.object_count,
                                os_.prims.size // 28, _p(views), views.shape[0], _p(pixels), pixels.size, _p(out),
                                threads, _p(tapes), tapes.shape[1])
    assert rc == 0
    return out


RULE_VISIBILITY, RULE_REPROJECTION = 1, 2


def set_reference_rules(rules: int, track: bool = False):
    """Reference rules of the oracle's shading, for the pin against the reference's own code only
    (pathtrace.cpp): RULE_VISIBILITY = the reference's closest-hit light test instead of the
    contract's any-hit; RULE_REPROJECTION = temporal reprojection through the float matrix the pin
    hands the reference. 0 = the contract (what the CUDA path does). With track, every light test
    also evaluates the other visibility rule. Returns (tests, disagreements) since the last call."""
    counts = np.zeros(2, np.uint64)
    _bind("oracle_set_reference_rules", [C.c_int, C.c_int, _P])(int(rules), int(track), _p(counts))
    return int(counts[0]), int(counts[1])


def light_tables(os_: "OracleScene", materials):
    """(indices, cdf, total, pdf per primitive) of the resident emissive primitives."""
    lib = load()
    if not hasattr(lib, "_lights_bound"):
        lib.oracle_light_tables.argtypes = [_P, _P, _P, _P, _P, C.c_uint32, _P, _P, _P, _P]
        lib.oracle_light_tables.restype = C.c_uint32
        lib._lights_bound = True
    n = os_.prims.size // 28
    idx, cdf, pdf = np.zeros(n, np.uint32), np.zeros(n, np.float32), np.zeros(n, np.float32)
    total = np.zeros(1, np.float32)
    k = lib.oracle_light_tables(_p(os_.prims), _p(np.ascontiguousarray(materials, np.float32)), _p(os_.active),
                                _p(os_.blas_root), _p(os_.prim_object), n, _p(idx), _p(cdf), _p(total), _p(pdf))
    return idx[:k].copy(), cdf[:k].copy(), float(total[0]), pdf


def _bind(name, argtypes):
    lib = load()
    fn = getattr(lib, name)
    if not getattr(fn, "_bound", False):
        fn.argtypes, fn.restype, fn._bound = argtypes, None, True
    return fn


def _c(a, dt, cols=None):
    a = np.ascontiguousarray(a, dt)
    return a if cols is None else a.reshape(-1, cols)


def decode_material(mats, lod=1.0):
    """decode() of each packed material: 17 floats (ref_decode_material's first 17)."""
    mats = _c(mats, np.float32, 20)
    out = np.zeros((mats.shape[0], 17), np.float32)
    _bind("oracle_decode_material", [_P, C.c_uint32, C.c_float, _P])(_p(mats), mats.shape[0], lod, _p(out))
    return out


def bsdf(mats, nvl):
    mats, nvl = _c(mats, np.float32, 20), _c(nvl, np.float32, 9)
    out = np.zeros((nvl.shape[0], 3), np.float32)
    _bind("oracle_bsdf", [_P, _P, C.c_uint32, _P])(_p(mats), _p(nvl), nvl.shape[0], _p(out))
    return out


def select_light(xi, cdf, total):
    xi, cdf = _c(xi, np.float32), _c(cdf, np.float32)
    off, pdf = np.zeros(xi.size, np.uint32), np.zeros(xi.size, np.float32)
    _bind("oracle_select_light", [_P, C.c_uint32, _P, C.c_uint32, C.c_float, _P, _P])(
        _p(xi), xi.size, _p(cdf), cdf.size, float(total), _p(off), _p(pdf))
    return off, pdf


def sample_light_point(prims, uv):
    prims, uv = _c(prims, np.float32, 28), _c(uv, np.float32, 2)
    out, ok = np.zeros((uv.shape[0], 7), np.float32), np.zeros(uv.shape[0], np.uint8)
    _bind("oracle_light_point", [_P, _P, C.c_uint32, _P, _P])(_p(prims), _p(uv), uv.shape[0], _p(out), _p(ok))
    return out, ok


def scatter(dn, front, mats, tape4):
    dn, mats, tape4 = _c(dn, np.float32, 6), _c(mats, np.float32, 20), _c(tape4, np.float32, 4)
    n = dn.shape[0]
    d, w, k = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.uint32)
    _bind("oracle_scatter", [_P, _P, _P, _P, C.c_uint32, _P, _P, _P])(
        _p(dn), _p(_c(front, np.uint8)), _p(mats), _p(tape4), n, _p(d), _p(w), _p(k))
    return d, w, k


def reservoir_chain(cand, xi):
    chains, k = xi.shape
    cand, xi = _c(cand, np.float32, 16), _c(xi, np.float32)
    out = np.zeros((chains, 18), np.float32)
    _bind("oracle_reservoir_chain", [_P, _P, C.c_uint32, C.c_uint32, _P])(_p(cand), _p(xi), chains, k, _p(out))
    return out


class RestirOracle:
    """Chains oracle_render_restir over consecutive frames (keeps the previous frame's
    reservoirs, surfaces and views). With tapes (reference mode only), render(views, tapes)
    draws each path's random numbers from tapes[path] in the reference's order."""

    def __init__(self, os_, materials, candidates=32, temporal=True, spatial=3, radius_px=30.0, m_cap=20.0,
                 reference_mode=False):
        lib = load()
        if not hasattr(lib, "_restir_bound"):
            lib.oracle_render_restir.argtypes = [_P, _P, C.c_uint32, _P, _P, _P, _P, _P, _P, C.c_uint32,
                                                 C.c_uint32, _P, C.c_uint32, _P, _P, _P, _P, _P, C.c_int,
                                                 _P, _P, _P, _P, C.c_uint32]
            lib.oracle_render_restir.restype = C.c_int
            lib.oracle_render_restir_tape.argtypes = lib.oracle_render_restir.argtypes + [_P, C.c_uint32]
            lib.oracle_render_restir_tape.restype = C.c_int
            lib._restir_bound = True
        self.os_ = os_
        self.mats = np.ascontiguousarray(materials, np.float32)
        self.cfg_u = np.array([candidates, int(temporal), spatial, int(reference_mode)], np.uint32)
        self.cfg_f = np.array([radius_px, m_cap], np.float32)
        self.prev = None

    def render(self, views, tapes=None):
        lib = load()
        os_ = self.os_
        views = np.ascontiguousarray(views).reshape(-1)
        P = int((views["width"].astype(np.int64) * views["height"] * views["spp"]).sum())
        npx = int((views["width"].astype(np.int64) * views["height"]).sum())
        resv = np.zeros((P, 12), np.float32)
        surf = np.zeros((P, 12), np.float32)
        rgb = np.zeros((npx, 3), np.float32)
        stats = np.zeros(4, np.uint64)
        have = self.prev is not None and self.prev[2].shape == views.shape and all(
            (self.prev[2][k] == views[k]).all() for k in ("width", "height", "spp"))
        pr, ps, pv = self.prev if have else (resv, surf, views)
        args = (_p(os_.bvh), _p(os_.tlas), os_.tlas.size // 8, _p(os_.prims), _p(self.mats), _p(os_.prim_indices),
                _p(os_.active), _p(os_.blas_root), _p(os_.prim_object), os_.object_count, os_.prims.size // 28,
                _p(views), views.shape[0], _p(self.cfg_u), _p(self.cfg_f), _p(pr), _p(ps),
                _p(np.ascontiguousarray(pv)), int(have), _p(resv), _p(surf), _p(rgb), _p(stats), 0)
        if tapes is None:
            rc = lib.oracle_render_restir(*args)
        else:
            tapes = np.ascontiguousarray(tapes, np.float32)
            assert tapes.shape[0] == P
            rc = lib.oracle_render_restir_tape(*args, _p(tapes), tapes.shape[1])
        assert rc == 0
        self.prev = (resv, surf, views.copy())
        self.last = (resv, surf)
        return rgb, stats


def compact(sb, active):
    """Compacted resident arrays of the reference's compacted residency path (compact.cpp) for
    the per-primitive mask `active`, trimmed to their lengths."""
    lib = load()
    if not hasattr(lib, "_compact_bound"):
        lib.oracle_compact.argtypes = [_P, C.c_uint32, _P, _P, _P, C.c_uint32, _P, C.c_uint32, _P, _P, _P,
                                       _P, _P, _P, _P, _P, _P]
        lib.oracle_compact.restype = C.c_int
        lib._compact_bound = True
    n, nn, nobj = int(sb.prim_count), int(sb.bvh_nodes.size // 8), int(sb.object_count)
    bvh = np.ascontiguousarray(sb.bvh_nodes, np.float32)
    prims = np.ascontiguousarray(sb.prims, np.float32)
    mats = np.ascontiguousarray(sb.materials, np.float32)
    idx = np.ascontiguousarray(sb.prim_indices, np.int32)
    inst = np.ascontiguousarray(sb.instances.view(np.int32).reshape(-1))
    act = np.ascontiguousarray(active, np.uint8)
    o_bvh = np.zeros(max(nn, 1) * 8, np.float32)
    o_prims = np.zeros(n * 28, np.float32)
    o_mats = np.zeros(n * 20, np.float32)
    o_idx = np.zeros(n, np.int32)
    o_remap = np.zeros(n, np.uint32)
    o_p2r = np.zeros(n, np.int32)
    o_inst = np.zeros(nobj * 4, np.int32)
    counts = np.zeros(2, np.uint32)
    assert lib.oracle_compact(_p(bvh), nn, _p(prims), _p(mats), _p(idx), n, _p(inst), nobj, _p(act),
                              _p(o_bvh), _p(o_prims), _p(o_mats), _p(o_idx), _p(o_remap), _p(o_p2r),
                              _p(o_inst), _p(counts)) == 0
    p, nodes = int(counts[0]), int(counts[1])
    return {"prim_count": p, "bvh_node_count": nodes, "bvh_nodes": o_bvh[: nodes * 8], "prims": o_prims[: p * 28],
            "materials": o_mats[: p * 20], "prim_indices": o_idx[:p], "remap": o_remap[:p],
            "prim_to_resident": o_p2r, "instances": o_inst.view(sb.instances.dtype)}
