"""Seeded ray sets for the parity tests (host numpy)."""
import numpy as np

from nomad_b200.native import RAY_DTYPE


def _pack(o, d, tmax=None):
    o = np.asarray(o, np.float32)
    d = np.asarray(d, np.float32)
    r = np.empty(o.shape[0], RAY_DTYPE)
    r["ox"], r["oy"], r["oz"] = o[:, 0], o[:, 1], o[:, 2]
    r["tmin"] = np.float32(1e-4)
    r["dx"], r["dy"], r["dz"] = d[:, 0], d[:, 1], d[:, 2]
    r["tmax"] = np.float32(np.inf) if tmax is None else np.asarray(tmax, np.float32)
    return r


def _norm(v):
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def tri_vertices(sb):
    p = sb.prims.reshape(-1, 7, 4)
    return p[:, 0, :3], p[:, 1, :3], p[:, 2, :3], p[:, 0, 3].astype(np.int32)


def aimed_rays(sb, n, seed, spread=1.5):
    """Rays from random points around the scene toward random points on random primitives."""
    rng = np.random.default_rng(seed)
    v0, v1, v2, _ = tri_vertices(sb)
    lo = sb.object_bounds.reshape(-1, 6)[:, :3].min(0)
    hi = sb.object_bounds.reshape(-1, 6)[:, 3:].max(0)
    c, ext = (lo + hi) / 2, (hi - lo) / 2 * spread
    o = c + (rng.random((n, 3)) * 2 - 1) * ext
    k = rng.integers(0, v0.shape[0], n)
    a, b = rng.random(n), rng.random(n)
    flip = a + b > 1
    a[flip], b[flip] = 1 - a[flip], 1 - b[flip]
    tgt = v0[k] + a[:, None] * (v1[k] - v0[k]) + b[:, None] * (v2[k] - v0[k])
    return _pack(o, _norm(tgt - o))


def random_rays(sb, n, seed):
    rng = np.random.default_rng(seed)
    lo = sb.object_bounds.reshape(-1, 6)[:, :3].min(0)
    hi = sb.object_bounds.reshape(-1, 6)[:, 3:].max(0)
    o = lo + rng.random((n, 3)) * (hi - lo)
    return _pack(o, _norm(rng.normal(size=(n, 3))))


def edge_case_rays(sb, seed):
    """Axis-parallel and near-parallel rays (|d| < 1e-4 on some axes), rays through shared
    triangle edges and vertices (exact-t ties), finite tmax, and rays starting on surfaces."""
    rng = np.random.default_rng(seed)
    v0, v1, v2, types = tri_vertices(sb)
    tri = np.nonzero(types == 1)[0]
    lo = sb.object_bounds.reshape(-1, 6)[:, :3].min(0)
    hi = sb.object_bounds.reshape(-1, 6)[:, 3:].max(0)
    span = float((hi - lo).max())
    out = []
    # axis-aligned rays toward triangle centroids from outside the scene
    k = rng.choice(tri, 600)
    cen = (v0[k] + v1[k] + v2[k]) / 3
    for ax in range(3):
        for sgn in (-1.0, 1.0):
            d = np.zeros((k.size, 3), np.float32)
            d[:, ax] = sgn
            o = cen - d * span
            out.append(_pack(o, d))
    # near-parallel: one component tiny (below and above the 1e-4 threshold)
    for tiny in (5e-5, 9.99e-5, 1.0e-4, 2e-4):
        d = rng.normal(size=(k.size, 3)).astype(np.float32)
        d[:, rng.integers(0, 3)] = tiny * np.sign(rng.normal(size=k.size))
        d = _norm(d)
        out.append(_pack(cen - d * span * 0.5, d))
    # through shared edges (midpoints) and vertices: exact ties in t between neighbours
    mid = (v0[k] + v1[k]) / 2
    d = _norm(rng.normal(size=(k.size, 3)))
    out.append(_pack(mid - d * span * 0.25, d))
    out.append(_pack(v2[k] - d * span * 0.25, d))
    # finite tmax around the hit distance
    d = _norm(rng.normal(size=(k.size, 3)))
    o = cen - d * 10.0
    out.append(_pack(o, d, tmax=np.float32(10.0) * rng.uniform(0.9, 1.1, k.size)))
    # origins on surfaces (self-intersection region) and zero tmax
    d = _norm(rng.normal(size=(k.size, 3)))
    out.append(_pack(cen, d))
    out.append(_pack(cen - d, d, tmax=np.zeros(k.size, np.float32)))
    return np.concatenate(out)
