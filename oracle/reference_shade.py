"""ORACLE — test infrastructure only.

ctypes wrapper of oracle/_ref/libref_shade.so: the reference's own shading code
(Renderer/Shaders/PathTraceKernel.metal with PathTracing.h and Scatter.h, compiled as C++ through
oracle/ref/shim/metal_compat.h by `make -C oracle ref`) run on the host with caller-supplied
random numbers ("tapes"; see oracle/ref/ref_shade.cpp). Each function takes the same arguments as
its counterpart in oracle.py (the contract oracle), so the two can be compared case by case.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libref_shade.so")
_lib = None
_P = C.c_void_p
U32, F32 = C.c_uint32, C.c_float


def available() -> bool:
    return os.path.exists(LIB_PATH)


def load():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle ref` where the reference exists")
        lib = C.CDLL(LIB_PATH)
        lib.ref_render_frame.argtypes = [_P, U32, _P, U32, _P, _P, _P, _P, _P, _P, U32, _P, _P, U32, F32, _P, _P, _P,
                                         _P, _P, _P, _P, U32, _P, U32]
        lib.ref_render_frame.restype = C.c_int
        lib.ref_decode_material.argtypes = [_P, U32, F32, _P]
        lib.ref_bsdf.argtypes = [_P, _P, U32, _P]
        lib.ref_select_light.argtypes = [_P, U32, _P, U32, F32, _P, _P]
        lib.ref_sample_light_point.argtypes = [_P, _P, U32, _P, _P]
        lib.ref_scatter.argtypes = [_P, _P, _P, _P, U32, _P, _P, _P]
        lib.ref_reservoir_chain.argtypes = [_P, _P, U32, U32, _P]
        for f in ("ref_decode_material", "ref_bsdf", "ref_select_light", "ref_sample_light_point", "ref_scatter",
                  "ref_reservoir_chain"):
            getattr(lib, f).restype = None
        _lib = lib
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data


def _c(a, dt):
    return np.ascontiguousarray(a, dt)


def render_frame(os_, materials, view, lights, tapes, restir=(0, 0, 0), prev_view=None, prev_tex=None,
                 threads=0):
    """One frame of the reference's pathTraceKernel over every pixel of one view.

    lights: (indices, cdf, total, pdf_of_prim) as oracle.light_tables returns them.
    tapes: float32 [pixels, T]. restir: (enabled, candidates, temporal reuse).
    Returns (rgb [pixels, 3], ReSTIR textures [5, pixels, 4] or None)."""
    lib = load()
    view = np.ascontiguousarray(view).reshape(-1)[:1]
    w, h = int(view["width"][0]), int(view["height"][0])
    tapes = _c(tapes, np.float32)
    assert tapes.shape[0] == w * h
    idx, cdf, total, pdf = lights
    rgb = np.zeros((w * h, 3), np.float32)
    tex = np.zeros((5, w * h, 4), np.float32) if restir[0] else None
    rs = np.asarray(restir, np.uint32)
    pv = None if prev_view is None else np.ascontiguousarray(prev_view).reshape(-1)[:1]
    pt = None if prev_tex is None else _c(prev_tex, np.float32)
    rc = lib.ref_render_frame(_p(os_.bvh), os_.bvh.size // 8, _p(os_.tlas), os_.tlas.size // 8, _p(os_.prims),
                              _p(_c(materials, np.float32)), _p(os_.prim_indices), _p(os_.active),
                              _p(os_.blas_root), _p(os_.prim_object), os_.prims.size // 28, _p(_c(idx, np.uint32)),
                              _p(_c(cdf, np.float32)), len(idx), float(total), _p(_c(pdf, np.float32)), _p(view),
                              _p(pv), _p(rs), _p(pt), _p(tex), _p(tapes), tapes.shape[1], _p(rgb), threads)
    assert rc == 0, rc
    return rgb, tex


def decode_material(mats, lod=1.0):
    lib = load()
    mats = _c(mats, np.float32).reshape(-1, 20)
    out = np.zeros((mats.shape[0], 20), np.float32)
    lib.ref_decode_material(_p(mats), mats.shape[0], lod, _p(out))
    return out


def bsdf(mats, nvl):
    lib = load()
    mats, nvl = _c(mats, np.float32).reshape(-1, 20), _c(nvl, np.float32).reshape(-1, 9)
    out = np.zeros((nvl.shape[0], 3), np.float32)
    lib.ref_bsdf(_p(mats), _p(nvl), nvl.shape[0], _p(out))
    return out


def select_light(xi, cdf, total):
    lib = load()
    xi, cdf = _c(xi, np.float32), _c(cdf, np.float32)
    off = np.zeros(xi.size, np.uint32)
    pdf = np.zeros(xi.size, np.float32)
    lib.ref_select_light(_p(xi), xi.size, _p(cdf), cdf.size, float(total), _p(off), _p(pdf))
    return off, pdf


def sample_light_point(prims, uv):
    lib = load()
    prims, uv = _c(prims, np.float32).reshape(-1, 28), _c(uv, np.float32).reshape(-1, 2)
    out = np.zeros((uv.shape[0], 7), np.float32)
    ok = np.zeros(uv.shape[0], np.uint8)
    lib.ref_sample_light_point(_p(prims), _p(uv), uv.shape[0], _p(out), _p(ok))
    return out, ok


def scatter(dn, front, mats, tape4):
    lib = load()
    dn, mats, tape4 = (_c(dn, np.float32).reshape(-1, 6), _c(mats, np.float32).reshape(-1, 20),
                       _c(tape4, np.float32).reshape(-1, 4))
    n = dn.shape[0]
    d, w, k = np.zeros((n, 3), np.float32), np.zeros((n, 3), np.float32), np.zeros(n, np.uint32)
    lib.ref_scatter(_p(dn), _p(_c(front, np.uint8)), _p(mats), _p(tape4), n, _p(d), _p(w), _p(k))
    return d, w, k


def reservoir_chain(cand, xi):
    lib = load()
    chains, k = xi.shape
    cand, xi = _c(cand, np.float32).reshape(chains * k, 16), _c(xi, np.float32)
    out = np.zeros((chains, 18), np.float32)
    lib.ref_reservoir_chain(_p(cand), _p(xi), chains, k, _p(out))
    return out
