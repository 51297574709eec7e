"""Host-side ray batches for the trace entry points (numpy).

Primary rays follow the reference's pinhole set-up: populateViewportUniforms
(Nomad Path Tracer/Renderer/Renderer.cpp:1237-1259) and the per-sample jitter of
pathTraceKernel (Renderer/Shaders/PathTraceKernel.metal:67-93). Bounce rays leave the hit
point offset by RAY_EPS along the normal facing the incoming ray (PathTracing.h:1857-1859)
with a cosine-weighted direction (Scatter.h:324-342).
"""
from __future__ import annotations

import numpy as np

from .native import RAY_DTYPE, HIT_DTYPE

RAY_EPS = np.float32(1e-4)


def _norm(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


class Camera:
    """Pinhole camera with the reference's viewport conventions (vertical fov in degrees)."""

    def __init__(self, position, look_at, up=(0.0, 1.0, 0.0), vfov=60.0, width=640, height=360):
        self.position = np.asarray(position, np.float32)
        self.look_at = np.asarray(look_at, np.float32)
        self.up = np.asarray(up, np.float32)
        self.vfov = float(vfov)
        self.width, self.height = int(width), int(height)
        forward = _norm(self.look_at - self.position)
        aspect = np.float32(self.width / self.height)
        half_h = np.float32(np.tan(np.float32(self.vfov * np.pi / 180.0) * 0.5))
        half_w = aspect * half_h
        w = _norm(-forward)
        u = _norm(np.cross(self.up, w))
        v = np.cross(w, u)
        self.viewport_u = (u * (2.0 * half_w)).astype(np.float32)
        self.viewport_v = (-v * (2.0 * half_h)).astype(np.float32)
        self.first_pixel = (self.position - w - self.viewport_u * 0.5 - self.viewport_v * 0.5).astype(np.float32)

    def primary_rays(self, spp: int = 1, seed: int = 0, jitter: bool = True) -> np.ndarray:
        """width*height*spp rays, pixel-major then sample."""
        W, H = self.width, self.height
        ys, xs = np.meshgrid(np.arange(H, dtype=np.float32), np.arange(W, dtype=np.float32), indexing="ij")
        ux = ((xs + 0.5) / W).reshape(-1, 1).repeat(spp, 1).reshape(-1)
        uy = ((ys + 0.5) / H).reshape(-1, 1).repeat(spp, 1).reshape(-1)
        n = ux.size
        if jitter:
            rng = np.random.default_rng(seed)
            ux = ux + ((rng.random(n, dtype=np.float32) - 0.5) / W)
            uy = uy + ((rng.random(n, dtype=np.float32) - 0.5) / H)
        d = (self.first_pixel[None, :] + ux[:, None] * self.viewport_u[None, :]
             + uy[:, None] * self.viewport_v[None, :]) - self.position[None, :]
        d = _norm(d.astype(np.float32)).astype(np.float32)
        rays = np.empty(n, RAY_DTYPE)
        rays["ox"], rays["oy"], rays["oz"] = self.position
        rays["tmin"] = RAY_EPS
        rays["dx"], rays["dy"], rays["dz"] = d[:, 0], d[:, 1], d[:, 2]
        rays["tmax"] = np.float32(np.inf)
        return rays


def hit_normals(prims: np.ndarray, hits: np.ndarray) -> np.ndarray:
    """Stored shading normals (packed float4 #6) of the hit primitives."""
    p = prims.reshape(-1, 7, 4)
    return p[hits["prim"], 6, :3].astype(np.float32)


def bounce_rays(rays: np.ndarray, hits: np.ndarray, prims: np.ndarray, seed: int = 1) -> np.ndarray:
    """One cosine-weighted diffuse bounce ray per hit ray (misses dropped)."""
    m = hits["prim"] >= 0
    r, h = rays[m], hits[m]
    o = np.stack([r["ox"], r["oy"], r["oz"]], 1)
    d = np.stack([r["dx"], r["dy"], r["dz"]], 1)
    p = (o + h["t"][:, None] * d).astype(np.float32)
    n = _norm(hit_normals(prims, h))
    flip = (n * d).sum(1) > 0
    n[flip] = -n[flip]
    rng = np.random.default_rng(seed)
    u1 = rng.random(p.shape[0], dtype=np.float32)
    u2 = rng.random(p.shape[0], dtype=np.float32)
    rr = np.sqrt(u1)
    th = np.float32(2 * np.pi) * u2
    up = np.where(np.abs(n[:, 2:3]) < 0.999, np.array([[0, 0, 1]], np.float32), np.array([[0, 1, 0]], np.float32))
    t = _norm(np.cross(up, n))
    b = _norm(np.cross(n, t))
    local = t * (rr * np.cos(th))[:, None] + b * (rr * np.sin(th))[:, None] + n * np.sqrt(np.maximum(0, 1 - u1))[:, None]
    dd = _norm(local).astype(np.float32)
    org = (p + RAY_EPS * n).astype(np.float32)
    out = np.empty(p.shape[0], RAY_DTYPE)
    out["ox"], out["oy"], out["oz"] = org[:, 0], org[:, 1], org[:, 2]
    out["tmin"] = RAY_EPS
    out["dx"], out["dy"], out["dz"] = dd[:, 0], dd[:, 1], dd[:, 2]
    out["tmax"] = np.float32(np.inf)
    return out


def shadow_rays(rays: np.ndarray, hits: np.ndarray, prims: np.ndarray, materials: np.ndarray,
                seed: int = 1) -> np.ndarray:
    """One shadow ray per hit ray (misses dropped), as the path tracer's next-event estimation
    casts them: from the hit point offset 5e-4 along the normal toward a uniformly drawn point on
    a uniformly drawn emissive primitive, tmax = distance - 1e-4 (any-hit queries)."""
    g = prims.reshape(-1, 28)
    m = materials.reshape(-1, 20)
    lum = m[:, 8] * 0.2126 + m[:, 9] * 0.7152 + m[:, 10] * 0.0722
    emissive = np.nonzero(m[:, 11] * lum > 0)[0]
    keep = hits["prim"] >= 0
    r, h = rays[keep], hits[keep]
    o = np.stack([r["ox"], r["oy"], r["oz"]], 1)
    d = np.stack([r["dx"], r["dy"], r["dz"]], 1)
    p = (o + h["t"][:, None] * d).astype(np.float32)
    n = _norm(hit_normals(prims, h))
    flip = (n * d).sum(1) > 0
    n[flip] = -n[flip]
    rng = np.random.default_rng(seed)
    e = emissive[rng.integers(0, emissive.shape[0], p.shape[0])]
    u1 = rng.random(p.shape[0], dtype=np.float32)
    u2 = rng.random(p.shape[0], dtype=np.float32)
    a, b, c = g[e, 0:3], g[e, 4:7], g[e, 8:11]
    tri = g[e, 3] == 1
    su = np.sqrt(u1)[:, None]
    q_tri = a * (1 - su) + b * (su * (1 - u2[:, None])) + c * (su * u2[:, None])
    q_rect = a + (2 * u1[:, None] - 1) * b + (2 * u2[:, None] - 1) * c
    q = np.where(tri[:, None], q_tri, q_rect).astype(np.float32)
    org = (p + np.float32(5e-4) * n).astype(np.float32)
    to = q - org
    dist = np.linalg.norm(to, axis=1)
    ok = dist > 2e-4
    out = np.empty(int(ok.sum()), RAY_DTYPE)
    dd = (to[ok] / dist[ok, None]).astype(np.float32)
    out["ox"], out["oy"], out["oz"] = org[ok, 0], org[ok, 1], org[ok, 2]
    out["tmin"] = RAY_EPS
    out["dx"], out["dy"], out["dz"] = dd[:, 0], dd[:, 1], dd[:, 2]
    out["tmax"] = (dist[ok] - np.float32(1e-4)).astype(np.float32)
    return out


def icosphere_camera(width=640, height=360) -> Camera:
    """Camera outside the 100 m cube of the icosphere scene, looking at its centre."""
    return Camera((0.0, 40.0, 170.0), (0.0, 0.0, 0.0), vfov=60.0, width=width, height=height)


def city_camera(width=1920, height=1080) -> Camera:
    """Elevated view over the 1 km city."""
    return Camera((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), vfov=60.0, width=width, height=height)
