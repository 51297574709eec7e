"""ORACLE — test infrastructure only.

Restatements used to check the device residency step and the learned scorer:
  * select(): the byte-budgeted selection of nomad_residency_step (restated from
    updateRayHitBudget, Nomad Path Tracer/Renderer/RendererResidency.cpp:2871-2946, per object
    under a byte budget: min_active first, then the visibility reserve, then greedy fill in
    (score desc, index asc) order, then toggles in index order up to max_toggles);
  * rayhit_keys(): the decayed-score adjustment of :2833-2840;
  * mlp_forward(): the 24 -> 128 -> 128 -> 1 ReLU MLP in float64 with the inputs and the
    hidden activations rounded to bfloat16 where the device rounds them.
"""
import math

import numpy as np


def rayhit_keys(score, hits, visible, memory_pressure):
    key = score.astype(np.float32).copy()
    vis = visible.astype(bool)
    lerp = np.float32(0.5) + (np.float32(0.2) - np.float32(0.5)) * np.float32(memory_pressure)
    off = ~vis
    key[off & (hits == 0)] = 0.0
    key[off & (hits != 0)] *= lerp
    key[vis & (key <= 0)] = 1.0
    return key


def select(keys, visible, nbytes, budget, reserve, min_active, current, max_toggles=0, always=False,
           resident_bonus=0.0):
    n = keys.shape[0]
    kk = np.asarray(keys, np.float32).copy()
    if resident_bonus:
        # hysteresis: a resident object's key k becomes k + bonus * |k| (float32, no fused ops)
        m = np.asarray(current).astype(bool)
        with np.errstate(all="ignore"):
            kk[m] = kk[m] + np.float32(resident_bonus) * np.abs(kk[m])
    k = np.where(np.isfinite(kk), kk, 0.0).astype(np.float32)
    if always:
        k = np.ones(n, np.float32)
    order = sorted(range(n), key=lambda i: (-float(k[i]), i))
    desired = np.zeros(n, np.uint8)
    used = 0
    unlimited = budget == 0 or always
    for o in order[:min_active]:
        desired[o] = 1
        used += int(nbytes[o])
    promoted = 0
    for o in order:
        if promoted >= reserve:
            break
        if not visible[o]:
            continue
        promoted += 1
        if desired[o]:
            continue
        if unlimited or used + int(nbytes[o]) <= budget:
            desired[o] = 1
            used += int(nbytes[o])
    for o in order:
        if desired[o]:
            continue
        if unlimited or used + int(nbytes[o]) <= budget:
            desired[o] = 1
            used += int(nbytes[o])
    res = current.astype(np.uint8).copy()
    toggles = 0
    for o in range(n):
        if desired[o] == res[o]:
            continue
        if max_toggles and toggles >= max_toggles:
            break
        res[o] = desired[o]
        toggles += 1
    return res, toggles


def reserve_count(n, base, motion_w, motion):
    m = min(max(motion, 0.0), 1.0)
    return int(min(n, math.ceil(n * (np.float32(base) + np.float32(motion_w) * np.float32(m)))))


def _bf16(x):
    """Round float32 values to bfloat16 (nearest even) and back."""
    x = np.asarray(x, np.float32)
    b = x.view(np.uint32).astype(np.uint64)
    lsb = (b >> 16) & 1
    r = ((b + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def mlp_forward(blob, feats):
    nf = 24
    o_w1, o_b1 = 0, 128 * 32
    o_w2 = o_b1 + 128
    o_b2 = o_w2 + 128 * 128
    o_w3 = o_b2 + 128
    o_b3 = o_w3 + 128
    o_mean = o_b3 + 1
    o_istd = o_mean + nf
    w1 = _bf16(blob[o_w1:o_b1].reshape(128, 32)[:, :nf]).astype(np.float64)
    b1 = blob[o_b1:o_w2].astype(np.float64)
    w2 = _bf16(blob[o_w2:o_b2].reshape(128, 128)).astype(np.float64)
    b2 = blob[o_b2:o_w3].astype(np.float64)
    w3 = blob[o_w3:o_b3].astype(np.float64)
    b3 = float(blob[o_b3])
    mean, istd = blob[o_mean:o_istd], blob[o_istd:o_istd + nf]
    x = _bf16((feats.astype(np.float32) - mean) * istd).astype(np.float64)
    h1 = _bf16(np.maximum(x @ w1.T + b1, 0.0).astype(np.float32)).astype(np.float64)
    h2 = np.maximum(h1 @ w2.T + b2, 0.0)
    return h2 @ w3 + b3


def _blob_parts(blob):
    nf = 24
    o = {"w1": 0, "b1": 128 * 32}
    o["w2"] = o["b1"] + 128
    o["b2"] = o["w2"] + 128 * 128
    o["w3"] = o["b2"] + 128
    o["b3"] = o["w3"] + 128
    o["mean"] = o["b3"] + 1
    o["istd"] = o["mean"] + nf
    return o


def mlp_gradient(blob, feats, targets):
    """Mean-squared-error gradient of the scorer over the samples, restated in float64 with the
    device's BF16 roundings (nomad_mlp_gradient / one training step, mlp.cu): BF16 standardised
    inputs, weights W1 and W2, hidden activations H1 and the gradients dZ2, dZ1 that enter a
    product; FP32 biases and output layer. Returns (gradient blob, loss)."""
    o = _blob_parts(blob)
    nf = 24
    B = feats.shape[0]
    w1 = _bf16(blob[o["w1"]:o["b1"]].reshape(128, 32)[:, :nf]).astype(np.float64)
    b1 = blob[o["b1"]:o["w2"]].astype(np.float64)
    w2 = _bf16(blob[o["w2"]:o["b2"]].reshape(128, 128)).astype(np.float64)
    b2 = blob[o["b2"]:o["w3"]].astype(np.float64)
    w3 = blob[o["w3"]:o["b3"]].astype(np.float64)
    b3 = float(blob[o["b3"]])
    mean, istd = blob[o["mean"]:o["istd"]], blob[o["istd"]:o["istd"] + nf]
    x = _bf16((feats.astype(np.float32) - mean) * istd).astype(np.float64)
    z1 = x @ w1.T + b1
    h1 = _bf16(np.maximum(z1, 0.0).astype(np.float32)).astype(np.float64)
    z2 = h1 @ w2.T + b2
    h2 = np.maximum(z2, 0.0)
    y = h2 @ w3 + b3
    d = y - targets.astype(np.float64)
    dy = 2.0 * d / B
    dz2 = np.where(z2 > 0, dy[:, None] * w3[None, :], 0.0)
    dz2b = _bf16(dz2.astype(np.float32)).astype(np.float64)
    dh1 = dz2b @ w2
    dz1 = np.where(z1 > 0, dh1, 0.0)
    dz1b = _bf16(dz1.astype(np.float32)).astype(np.float64)
    g = np.zeros(blob.size, np.float64)
    gw1 = np.zeros((128, 32))
    gw1[:, :nf] = dz1b.T @ x
    g[o["w1"]:o["b1"]] = gw1.reshape(-1)
    g[o["b1"]:o["w2"]] = dz1.sum(0)
    g[o["w2"]:o["b2"]] = (dz2b.T @ h1).reshape(-1)
    g[o["b2"]:o["w3"]] = dz2.sum(0)
    g[o["w3"]:o["b3"]] = (h2 * dy[:, None]).sum(0)
    g[o["b3"]] = dy.sum()
    return g, float((d * d).mean())


def adamw_step(blob, grad, m, v, step, lr, wd, b1=0.9, b2=0.999, eps=1e-8):
    """One AdamW step (k_adamw, mlp.cu) in float32 over the trainable part of the blob (everything
    before the feature statistics): decoupled weight decay on W1, W2 and w3, not on the biases.
    Returns (blob, m, v)."""
    o = _blob_parts(blob)
    f = np.float32
    n = o["mean"]
    p, g = blob[:n].astype(f).copy(), grad[:n].astype(f)
    m, v = m[:n].astype(f), v[:n].astype(f)
    mi = f(b1) * m + (f(1) - f(b1)) * g
    vi = f(b2) * v + (f(1) - f(b2)) * g * g
    bc1 = f(1) - np.power(f(b1), f(step))
    bc2 = f(1) - np.power(f(b2), f(step))
    mh, vh = mi / bc1, vi / bc2
    i = np.arange(n)
    weight = (i < o["b1"]) | ((i >= o["w2"]) & (i < o["b2"])) | ((i >= o["w3"]) & (i < o["b3"]))
    p = np.where(weight, p - f(lr) * f(wd) * p, p)
    p = p - f(lr) * mh / (np.sqrt(vh) + f(eps))
    out = blob.astype(f).copy()
    out[:n] = p
    return out, mi, vi


class RayHitPrimOracle:
    """updateRayHitBudget per primitive (RendererResidency.cpp:2755-2964) with the per-frame
    cooldown decrement (:205-207) and the score pass of processRayHitCounters, restated in numpy
    float32. The frustum test is checked separately (in_view_f64) and taken as given here."""

    def __init__(self, prim_count, active=None):
        self.n = prim_count
        self.score = np.zeros(prim_count, np.float32)
        self.cooldown = np.zeros(prim_count, np.uint32)
        self.active = np.ones(prim_count, np.uint8) if active is None else active.astype(np.uint8).copy()
        self.rebuild = 0

    def step(self, hits, visible, decay=0.85, motion=0.0, pressure=0.0, target_fraction=0.54, max_toggles=16,
             min_active=16, rebuild_cooldown=4, state_cooldown=5):
        f32 = np.float32
        n = self.n
        self.score = (self.score * f32(decay) + hits.astype(f32)).astype(f32)
        self.cooldown = np.where(self.cooldown > 0, self.cooldown - 1, 0).astype(np.uint32)
        self.ran = self.rebuild == 0
        if self.rebuild > 0:
            self.rebuild -= 1
            return 0
        m = f32(min(max(motion, 0.0), 1.0))
        p = f32(min(max(pressure, 0.0), 1.0))
        frac = f32(min(max(f32(target_fraction) + f32(0.10) * m - f32(0.24) * p, f32(0.34)), f32(0.92)))
        unlimited = max_toggles == 0
        budget = max(1, int(np.floor(float(max(max_toggles, 1)) * (1.0 + 0.45 * float(m) + 0.60 * float(p)) + 0.5)))
        keep = f32(0.5) + (f32(0.2) - f32(0.5)) * p
        vis = visible.astype(bool)
        adj = self.score.copy()
        adj[~vis & (hits == 0)] = f32(0.0)
        sel = ~vis & (hits != 0)
        adj[sel] = (adj[sel] * keep).astype(f32)
        adj[vis & (adj <= 0)] = f32(1.0)
        big = np.finfo(np.float32).max
        adj = np.where(np.isnan(adj), -big, np.clip(adj, -big, big)).astype(f32)
        order = np.lexsort((np.arange(n), -adj.astype(np.float64)))
        min_active_n = min(n, min_active)
        target = int(np.ceil(f32(n) * frac))
        target = min(max(target, min_active_n), n)
        desired = np.zeros(n, bool)
        desired[order[:target]] = True
        reserve = min(n, int(np.ceil(f32(n) * (f32(0.02) + f32(0.06) * m))))
        vis_order = order[vis[order]][:reserve]
        desired[vis_order] = True
        desired[order[:min_active_n]] = True
        toggles = 0
        for i in np.nonzero(desired != self.active.astype(bool))[0]:
            if not unlimited:
                if self.cooldown[i] > 0:
                    continue
                if toggles >= budget:
                    break
            self.active[i] = 1 if desired[i] else 0
            self.cooldown[i] = state_cooldown
            toggles += 1
        if not self.active.any() and n > 0:
            self.active[order[0]] = 1
            self.cooldown[order[0]] = state_cooldown
            toggles += 1
        if toggles:
            self.rebuild = rebuild_cooldown
        return toggles


def in_view_f64(spheres, view):
    """Renderer::isInView (Renderer.cpp:1765-1817) in float64 with the view's camera; returns the
    test and each sphere's margin (radians) from the decision boundary."""
    v = np.asarray(view).reshape(-1)[0]
    pos = v["camera_pos"].astype(np.float64)
    U, V = v["viewport_u"].astype(np.float64), v["viewport_v"].astype(np.float64)
    f = v["first_pixel"].astype(np.float64) + 0.5 * U + 0.5 * V - pos
    fl = np.linalg.norm(f)
    fwd = f / fl
    up = -V / np.linalg.norm(V)
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    up /= np.linalg.norm(up)
    half_v = np.arctan(0.5 * np.linalg.norm(V) / fl)
    half_h = np.arctan(np.tan(half_v) * float(v["width"]) / float(v["height"]))
    c = spheres[:, :3].astype(np.float64) - pos
    dist = np.linalg.norm(c, axis=1)
    d = c / np.maximum(dist, 1e-30)[:, None]
    fd = d @ fwd
    ra = np.arcsin(np.minimum(spheres[:, 3] / np.maximum(dist, 1e-30), 1.0))
    h = np.arctan2(np.abs(d @ right), fd)
    vv = np.arctan2(np.abs(d @ up), fd)
    margin = np.minimum(half_h + ra - h, half_v + ra - vv)
    vis = (fd > 0) & (margin >= 0)
    vis |= dist < 1e-5
    margin = np.where(fd > 0, margin, np.abs(fd))
    return vis, np.abs(margin)


def prim_spheres(prims):
    """Renderer.cpp:3158-3173: spheres as they are; triangles around the centroid, radius the
    farthest vertex; rectangles around the centre, radius |u| + |v| (float64)."""
    g = prims.reshape(-1, 28).astype(np.float64)
    t = g[:, 3].astype(np.int32)
    out = np.zeros((g.shape[0], 4))
    v0, v1, v2 = g[:, 0:3], g[:, 4:7], g[:, 8:11]
    c = (v0 + v1 + v2) / 3.0
    r = np.maximum(np.maximum(np.linalg.norm(v0 - c, axis=1), np.linalg.norm(v1 - c, axis=1)),
                   np.linalg.norm(v2 - c, axis=1))
    tri = t == 1
    out[tri, :3], out[tri, 3] = c[tri], r[tri]
    sph = t == 0
    out[sph, :3], out[sph, 3] = v0[sph], g[sph, 4]
    rect = t == 2
    out[rect, :3] = v0[rect]
    out[rect, 3] = np.linalg.norm(v1[rect], axis=1) + np.linalg.norm(v2[rect], axis=1)
    return out


class DistanceLodOracle:
    """updateLODByDistance (RendererResidency.cpp:759-964) restated over the per-object distance
    and frustum flags of the step (checked separately by lod_tests_f64): nearest first (equal
    distances by index), hysteresis between the entry and exit distances and frusta, object
    cooldowns (:208-210, :1025), the toggle budget."""

    def __init__(self, object_count, prim_counts):
        self.n = object_count
        self.count = prim_counts.astype(np.int64)
        self.active_count = self.count.copy()
        self.cooldown = np.zeros(object_count, np.uint32)

    def step(self, dist, flags, motion=0.0, pressure=0.0, max_toggles=24, enter=225.0, exit_=275.0,
             state_cooldown=5):
        self.cooldown = np.where(self.cooldown > 0, self.cooldown - 1, 0).astype(np.uint32)
        m, p = min(max(motion, 0.0), 1.0), min(max(pressure, 0.0), 1.0)
        budget = max(1, int(np.floor(float(max(max_toggles, 1)) * (1.0 + 0.40 * np.float32(m) + 0.60 * np.float32(p))
                                     + 0.5)))
        order = np.lexsort((np.arange(self.n), dist.astype(np.float64)))
        toggles = 0
        for o in order:
            active = self.active_count[o] > 0
            view_ok = bool(flags[o] & 2) if active else bool(flags[o] & 1)
            behind = bool(flags[o] & 4)
            d = np.float32(dist[o])
            want = view_ok and not behind and (d <= np.float32(exit_) if active else d < np.float32(enter))
            if self.cooldown[o] != 0 or want == active:
                continue
            needed = self.count[o] - self.active_count[o] if want else self.active_count[o]
            if needed == 0:
                continue
            if toggles + 1 > budget:
                continue
            self.active_count[o] = self.count[o] if want else 0
            self.cooldown[o] = state_cooldown
            toggles += 1
        return toggles


def lod_tests_f64(spheres, view, enter_deg=5.0, exit_deg=12.0):
    """The per-object distance and entry/exit frustum tests of updateLODByDistance in float64;
    returns (distance, enter, exit, behind, angular margin of the nearer frustum boundary)."""
    v = np.asarray(view).reshape(-1)[0]
    pos = v["camera_pos"].astype(np.float64)
    U, V = v["viewport_u"].astype(np.float64), v["viewport_v"].astype(np.float64)
    f = v["first_pixel"].astype(np.float64) + 0.5 * U + 0.5 * V - pos
    fl = np.linalg.norm(f)
    fwd = f / fl
    up = -V / np.linalg.norm(V)
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    up /= np.linalg.norm(up)
    half_v = np.arctan(0.5 * np.linalg.norm(V) / fl)
    half_h = np.arctan(np.tan(half_v) * float(v["width"]) / float(v["height"]))
    em = np.radians(max(enter_deg, 0.0))
    xm = max(np.radians(max(exit_deg, 0.0)), em)
    t = spheres[:, :3] - pos
    dtc = np.linalg.norm(t, axis=1)
    r = spheres[:, 3]
    fd = t @ fwd
    behind = fd + r <= 0
    dist = np.where(behind, np.finfo(np.float32).max, np.maximum(dtc - r, 0.0))
    depth = np.maximum(fd, 1e-5)
    ha = np.arctan2(np.abs(t @ right), depth)
    va = np.arctan2(np.abs(t @ up), depth)
    ra = np.arcsin(np.minimum(r / np.maximum(dtc, 1e-30), 1.0))
    enter = (ha <= half_h + ra + em) & (va <= half_v + ra + em)
    exit_ = (ha <= half_h + ra + xm) & (va <= half_v + ra + xm)
    near = dtc <= 1e-5
    enter = np.where(near | behind, ~behind, enter)
    exit_ = np.where(near | behind, ~behind, exit_)
    margin = np.minimum.reduce([np.abs(half_h + ra + em - ha), np.abs(half_v + ra + em - va),
                                np.abs(half_h + ra + xm - ha), np.abs(half_v + ra + xm - va)])
    margin = np.where(near | behind, np.inf, margin)
    return dist, enter, exit_, behind, margin


def object_spheres(sb):
    """Each object's bounding sphere from its BLAS root box (Renderer.cpp:3272-3278), float32
    arithmetic as the library does it."""
    nodes = sb.bvh_nodes.reshape(-1, 8)
    roots = sb.instances["blas_root_index"]
    out = np.zeros((sb.object_count, 4), np.float32)
    for o, r in enumerate(roots):
        if r < 0:
            continue
        mn, mx = nodes[r, 0:3].astype(np.float32), nodes[r, 4:7].astype(np.float32)
        c = ((mn + mx) * np.float32(0.5)).astype(np.float32)
        d = (mx - c).astype(np.float32)
        out[o, :3] = c
        out[o, 3] = np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]), dtype=np.float32)
    return out


class ScreenSpaceOracle:
    """updateScreenSpaceFootprint (RendererResidency.cpp:4092-4396) with one mesh group per object,
    restated over the per-object coverage of the step (checked by coverage_f64): groups by
    coverage until min_active primitives and the target share of the screen are covered, toggles
    in coverage order under a primitive budget, object and primitive cooldowns (whole objects are
    toggled here, so one cooldown per object carries both)."""

    def __init__(self, prim_counts):
        self.count = prim_counts.astype(np.int64)
        self.n = self.count.size
        self.active = self.count > 0
        self.cooldown = np.zeros(self.n, np.uint32)

    def step(self, cov, width, height, motion=0.0, pressure=0.0, target_fraction=0.68, min_pixel=32.0,
             min_active=16, max_toggles=14, state_cooldown=5):
        f32 = np.float32
        self.cooldown = np.where(self.cooldown > 0, self.cooldown - 1, 0).astype(np.uint32)
        m, p = f32(min(max(motion, 0.0), 1.0)), f32(min(max(pressure, 0.0), 1.0))
        frac = f32(min(max(f32(target_fraction) + f32(0.08) * m - f32(0.10) * p, f32(0.50)), f32(0.94)))
        budget = max(1, int(np.floor(float(max(max_toggles, 1)) * (1.0 + 0.40 * float(m) + 0.50 * float(p)) + 0.5)))
        area = f32(width) * f32(height)
        if area <= 0:
            area = f32(1.0)
        order = np.lexsort((np.arange(self.n), -cov.astype(np.float64)))
        min_active_n = min(int(self.count.sum()), min_active)
        target = f32(area * frac)
        desired = np.zeros(self.n, bool)
        enabled, acc = 0, f32(0.0)
        for g in order:
            c = self.count[g]
            if c == 0:
                continue
            cv = f32(cov[g])
            min_sat, cov_sat = enabled >= min_active_n, acc >= target
            if min_sat and cov_sat:
                break
            if min_sat and cv < f32(min_pixel):
                continue
            if min_sat and cv <= 0:
                continue
            desired[g] = True
            enabled += c
            acc = f32(acc + cv)
        for g in order:
            if enabled >= min_active_n:
                break
            if desired[g] or self.count[g] == 0:
                continue
            desired[g] = True
            enabled += self.count[g]
            acc = f32(acc + f32(cov[g]))
        toggled = 0
        for g in order:
            if toggled >= budget:
                break
            if desired[g] == self.active[g] or self.cooldown[g] > 0 or self.count[g] == 0:
                continue
            self.active[g] = desired[g]
            self.cooldown[g] = state_cooldown
            toggled = min(toggled + int(self.count[g]), budget)
        return toggled


def coverage_f64(spheres, view):
    """objectCoverageForSphere (RendererResidency.cpp:4130-4182) in float64, with the margin of
    each decision (frustum, depth, horizontal angle) for the comparison."""
    vis, vmargin = in_view_f64(spheres.astype(np.float64), view)
    v = np.asarray(view).reshape(-1)[0]
    pos = v["camera_pos"].astype(np.float64)
    U, V = v["viewport_u"].astype(np.float64), v["viewport_v"].astype(np.float64)
    f = v["first_pixel"].astype(np.float64) + 0.5 * U + 0.5 * V - pos
    fl = np.linalg.norm(f)
    fwd = f / fl
    up = -V / np.linalg.norm(V)
    right = np.cross(fwd, up)
    right /= np.linalg.norm(right)
    tan_half = 0.5 * np.linalg.norm(V) / fl
    W, H = float(v["width"]), float(v["height"])
    h_half = np.arctan(tan_half * W / H)
    t = spheres[:, :3].astype(np.float64) - pos
    depth = t @ fwd
    dist = np.linalg.norm(t, axis=1)
    cos_a = depth / np.maximum(dist, 1e-3)
    ha = np.arctan2(np.abs(t @ right), depth)
    rp = np.maximum((spheres[:, 3] / depth) / tan_half * (H * 0.5), 0.0)
    cov = np.minimum(np.pi * rp * rp * np.maximum(cos_a, 0.0), W * H)
    ok = vis & (depth > 1e-3) & (ha <= h_half + 0.1)
    cov = np.where(ok, cov, 0.0)
    margin = np.minimum.reduce([vmargin, np.abs(depth - 1e-3), np.abs(h_half + 0.1 - ha)])
    return cov, margin


# ------------------------------------------------------------------------------------------------
# Per-object hit-probability posterior and the Probabilistic policy

def object_tests(os_, rays, t_hit):
    """Per-object "rays tested" (oracle_object_tests, contract.cpp): the resident objects whose
    TLAS leaf box each ray's segment [1e-4, t_hit] enters."""
    import ctypes as C
    from . import oracle as orc

    lib = orc.load()
    fn = lib.oracle_object_tests
    fn.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_uint64, C.c_void_p]
    fn.restype = C.c_int
    rays = np.ascontiguousarray(rays)
    t = np.ascontiguousarray(t_hit, np.float32)
    out = np.zeros(os_.object_count, np.uint32)
    assert fn(os_.tlas.ctypes.data, os_.tlas.size // 8, os_.blas_root.ctypes.data, os_.object_count,
              rays.ctypes.data, t.ctypes.data, rays.shape[0], out.ctypes.data) == 0
    return out


class ObjectPosterior:
    """processRayHitCounters' per-object Beta posterior (Renderer.cpp:8420-8522) in numpy float32,
    in the device kernel's operation order (k_posterior, residency.cu): alpha, beta, clamped
    probability, variance, mass, exploration score, idle steps."""

    def __init__(self, n):
        f = np.float32
        self.alpha = np.ones(n, f)
        self.beta = np.ones(n, f)
        self.probability = np.full(n, 0.5, f)
        self.variance = np.full(n, f(1.0) / f(12.0), f)
        self.mass = np.full(n, 2.0, f)
        self.exploration = np.zeros(n, f)
        self.idle = np.zeros(n, np.uint32)

    def step(self, hits, tests, visible, active, decay=0.9, hit_decay=0.85, window=64.0, idle_frames=0,
             idle_decay=0.9, threshold=0.5):
        f = np.float32
        decay, hit_decay, idle_decay, threshold = f(decay), f(hit_decay), f(idle_decay), f(threshold)
        clamp_mass = window > 0 and np.isfinite(window)
        max_mass = max(f(window), f(1.0e-3))
        visible, active = np.asarray(visible, bool), np.asarray(active, bool)
        success, rays = hits.astype(f), tests.astype(f)
        failure = np.maximum(rays - success, f(0))
        alpha = self.alpha * decay + success
        beta = self.beta * decay + failure
        s = alpha + beta
        with np.errstate(all="ignore"):
            prob = np.where(s > 0, alpha / s, f(0.5)).astype(f)
        idle = self.idle.copy()
        cool = tests == 0
        grace = (idle_frames > 0) & (visible | active) & (idle < idle_frames)
        factor = np.full(alpha.shape, decay, f)
        apply = cool.copy()
        if idle_decay >= f(0.999):
            apply &= ~grace
        else:
            factor = np.where(grace, idle_decay, factor).astype(f)
        cp = np.clip(prob * factor, f(0), f(1))
        cm = np.maximum(s, f(1.0e-3))
        if clamp_mass:
            cm = np.where(cm > max_mass, max_mass, cm).astype(f)
        alpha = np.where(apply, cp * cm, alpha).astype(f)
        beta = np.where(apply, np.maximum(cm - cp * cm, f(0)), beta).astype(f)
        # renormalise the mass into [1e-3, window]
        s = alpha + beta
        zero = ~(s > 0)
        small = (~zero) & (s < f(1.0e-3))
        with np.errstate(all="ignore"):
            scale = np.where(small, f(1.0e-3) / s, f(1)).astype(f)
        alpha = np.where(small, alpha * scale, alpha).astype(f)
        beta = np.where(small, beta * scale, beta).astype(f)
        alpha = np.where(zero, f(1.0e-3) * f(0.5), alpha).astype(f)
        beta = np.where(zero, f(1.0e-3) * f(0.5), beta).astype(f)
        s = np.where(zero | small, f(1.0e-3), s).astype(f)
        if clamp_mass:
            big = s > max_mass
            with np.errstate(all="ignore"):
                scale = np.where(big, max_mass / s, f(1)).astype(f)
            alpha = np.where(big, alpha * scale, alpha).astype(f)
            beta = np.where(big, beta * scale, beta).astype(f)
            s = np.where(big, max_mass, s).astype(f)
        with np.errstate(all="ignore"):
            prob = np.where(s > 0, alpha / s, f(0.5)).astype(f)
            var = np.where(s > 1, (alpha * beta) / ((s * s) * (s + f(1))), f(0)).astype(f)
        clamped = np.clip(prob, f(0), f(1))
        ex = self.exploration * decay
        tested = tests > 0
        ex = np.where(tested, np.where(clamped < threshold, ex + rays, ex * hit_decay), ex * hit_decay).astype(f)
        ex = np.where((~tested) & (visible | active), np.maximum(ex, f(1)), ex).astype(f)
        idle = np.where(tested, 0, np.minimum(idle.astype(np.uint64) + 1, 0xFFFFFFFF)).astype(np.uint32)
        self.alpha, self.beta, self.probability = alpha, beta, clamped
        self.variance, self.mass, self.exploration, self.idle = np.maximum(var, f(0)), s, ex, idle


def rayhit_prior(probability, scale):
    """The reference's ray-hit prior weight clamp(1 + (p - 0.5) * scale, 0.25, 1)
    (RendererResidency.cpp:2842-2861, favouring high probability off)."""
    f = np.float32
    w = f(1) + (probability.astype(f) - f(0.5)) * f(scale) * f(1)
    return np.clip(w, f(0.25), f(1)).astype(f)


class ProbabilisticOracle:
    """updateProbabilisticResidency's object-level path (RendererResidency.cpp:3389-4090), one
    object at a time (primitive counts are the objects'; their cooldowns are the object's), in
    numpy float32, over the posterior of the same step (ObjectPosterior, whose exploration scores
    it updates as the reference does). step() returns the object activity after the toggles."""

    def __init__(self, prim_counts):
        n = len(prim_counts)
        self.counts = np.asarray(prim_counts, np.int64)
        self.desired_state = np.zeros(n, np.uint8)
        self.pending = np.zeros(n, np.uint8)
        self.promoted = np.zeros(n, np.int64)
        self.demoted = np.zeros(n, np.int64)
        self.dwell = np.zeros(n, np.int64)
        self.evidence = np.zeros(n, np.float32)
        self.order = list(range(n))
        self.cooldown = np.zeros(n, np.int64)

    def decrement_cooldowns(self):
        self.cooldown = np.maximum(self.cooldown - 1, 0)

    def step(self, post, tests_last, visible, active, frame_no, target_fraction=0.60, min_active=16,
             max_toggles=20, camera_motion=0.0, memory_pressure=0.0, window=64.0, threshold=0.5,
             uncertainty_boost=0.25, desired_hysteresis=0.02, visible_floor=0.0, recent_promotion_frames=4,
             demotion_dwell_frames=0, state_cooldown=5):
        import math

        f = np.float32
        n = len(self.counts)
        active = np.asarray(active, bool).copy()
        vis = np.asarray(visible, bool)
        prim_count = int(self.counts.sum())
        contribution = np.maximum(self.counts, 1)

        def cl(v):
            return min(max(f(v), f(0)), f(1))

        motion, pressure = cl(camera_motion), cl(memory_pressure)
        tf = min(max(f(target_fraction) + f(0.08) * motion - f(0.12) * pressure, f(0.45)), f(0.93))
        base = max(int(max_toggles), 1)
        budget = max(1, int(math.floor(base * (1.0 + 0.40 * float(motion) + 0.50 * float(pressure)) + 0.5)))
        finite = window > 0 and np.isfinite(window)
        scoring = max(f(window), f(1e-3)) if finite else max(f(64.0), f(1e-3))
        thr = f(threshold)

        def evidence(mass, visible_):
            if not (mass > 0) or not np.isfinite(mass) or not visible_:
                return f(0)
            return cl(mass / scoring) if finite else cl(mass / (mass + scoring))

        def sane(p):
            return cl(p) if np.isfinite(p) else f(0.5)

        def regressed(p, e):
            ce = cl(e)
            return sane(p) * ce + f(0.5) * (f(1) - ce)

        def score_e(p, var, e):
            v = f(0) if (not np.isfinite(var) or var < 0) else f(var)
            return regressed(p, e) + f(uncertainty_boost) * np.sqrt(max(v, f(0)))

        P, V, M, X = post.probability, post.variance, post.mass, post.exploration
        desired = self.desired_state.copy()
        pending = self.pending
        hyst = min(max(f(desired_hysteresis), f(0)), f(0.5))
        enter_t, exit_t = cl(thr + hyst), cl(thr - hyst)
        floor_v = cl(visible_floor)
        desired_count = 0
        for i in range(n):
            raw = evidence(M[i], vis[i])
            buffered = max(cl(raw), self.evidence[i] * f(0.9))
            self.evidence[i] = buffered
            eff = regressed(sane(P[i]), buffered)
            boosted = score_e(P[i], V[i], buffered)
            enter_s, exit_s = max(eff, boosted), eff
            prev = bool(desired[i])
            want = prev
            low = min(buffered, cl(raw)) <= f(1e-3)
            promotion, demotion, evaluation = enter_s, exit_s, (eff if low else enter_s)
            dwell_applies = bool(vis[i]) and demotion_dwell_frames > 0
            if not dwell_applies or demotion > exit_t:
                self.dwell[i] = 0
            if vis[i]:
                demotion = max(demotion, floor_v)
                evaluation = max(evaluation, floor_v)
            if promotion >= enter_t:
                want = True
                self.dwell[i] = 0
            elif demotion <= exit_t:
                if dwell_applies and prev:
                    if self.dwell[i] < demotion_dwell_frames:
                        self.dwell[i] += 1
                    want = self.dwell[i] < demotion_dwell_frames
                else:
                    want = False
                    self.dwell[i] = 0
            elif self.cooldown[i] == 0 and not prev:
                want = evaluation >= thr
                if want:
                    self.dwell[i] = 0
            if want and not prev:
                self.promoted[i] = frame_no
            elif not want and prev:
                self.demoted[i] = frame_no
            desired[i] = 1 if want else 0
            if not want:
                pending[i] = 0
            if want and not pending[i]:
                desired_count += int(contribution[i])
        min_act = min(int(min_active), prim_count)
        keys = [_sanitize(score_e(P[o], V[o], evidence(M[o], vis[o]))) for o in range(n)]
        self.order.sort(key=lambda o: (-keys[o], o))
        order = self.order
        target = int(math.ceil(f(prim_count) * tf))
        target = max(target, min_act)
        if target == 0 and prim_count > 0:
            target = 1
        target = min(target, prim_count)

        def trim():
            nonlocal desired_count
            if target == 0 or desired_count <= target:
                return
            for idx in reversed(order):
                if desired_count <= target:
                    break
                if not desired[idx] or pending[idx]:
                    continue
                c = int(contribution[idx])
                desired[idx] = 0
                pending[idx] = 0
                self.demoted[idx] = frame_no
                desired_count = desired_count - c if desired_count > c else 0

        trim()
        vis_x, hid_x = [], []
        for idx in order:
            if active[idx] or desired[idx]:
                continue
            raw = evidence(M[idx], vis[idx])
            buffered = self.evidence[idx]
            eff = regressed(P[idx], buffered)
            low = min(buffered, cl(raw)) <= f(1e-3)
            gated = min(eff, thr) if (vis[idx] and low) else eff
            if gated > thr:
                continue
            rays = int(tests_last[idx])
            ex = f(X[idx])
            if vis[idx] and (rays == 0 or low):
                ex = max(ex, f(1))
            if vis[idx] and rays > 0 and not low:
                ex = max(ex, f(1e-3))
            X[idx] = ex
            if ex <= 0:
                continue
            (vis_x if vis[idx] else hid_x).append(idx)
        vis_x.sort(key=lambda o: (-_sanitize(X[o]), -int(tests_last[o]), o))
        hid_x.sort(key=lambda o: (-_sanitize(X[o]), -int(tests_last[o]), o))

        def recent(idx):
            w = recent_promotion_frames
            if w == 0:
                return False
            last = max(self.promoted[idx], self.demoted[idx])
            if last == 0:
                return False
            if frame_no <= last:
                return True
            return frame_no - last < w

        def mark(idx):
            nonlocal desired_count
            desired[idx] = 1
            self.promoted[idx] = frame_no
            c = int(contribution[idx])
            if not pending[idx]:
                desired_count += c
            if vis[idx] and int(tests_last[idx]) == 0 and X[idx] < f(1):
                X[idx] = f(1)
            return c

        def promote(cands, slots, allow):
            if slots == 0:
                return 0
            for idx in cands:
                if slots == 0:
                    break
                if desired[idx]:
                    continue
                if not allow and recent(idx):
                    continue
                c = mark(idx)
                slots = 0 if slots <= c else slots - c
            return slots

        def remaining_of(cands):
            return sum(int(contribution[i]) for i in cands if not desired[i] and not pending[i])

        if desired_count < min_act:
            slots = min(min_act - desired_count, prim_count - desired_count if prim_count > desired_count else 0)
            slots = promote(vis_x, slots, False)
            slots = promote(hid_x, slots, False)
            if slots > 0:
                slots = promote(vis_x, slots, True)
                slots = promote(hid_x, slots, True)
        if desired_count < min_act:
            for allow in (False, True):
                if desired_count >= min_act:
                    break
                for idx in order:
                    if desired_count >= min_act:
                        break
                    if desired[idx]:
                        continue
                    if not allow and recent(idx):
                        continue
                    mark(idx)
        remaining = remaining_of(vis_x) + remaining_of(hid_x)
        if remaining > 0 and desired_count < prim_count:
            slots = min(max(1, min_act // 2), remaining, prim_count - desired_count)
            slots = promote(vis_x, slots, False)
            slots = promote(hid_x, slots, False)
            if slots > 0:
                slots = promote(vis_x, slots, True)
                slots = promote(hid_x, slots, True)
        desired_count = sum(int(contribution[i]) for i in range(n) if desired[i] and not pending[i])
        trim()
        fallback = vis_x[0] if vis_x else (hid_x[0] if hid_x else (order[0] if order else n))

        def set_object(o, want):
            prev_state = bool(active[o])
            toggled = int(self.counts[o]) if (want != prev_state) else 0
            active[o] = want and self.counts[o] > 0
            new_state = bool(active[o])
            self.desired_state[o] = 1 if new_state else 0
            if new_state:
                self.promoted[o] = frame_no
            else:
                self.demoted[o] = frame_no
            if not new_state or toggled > 0:
                pending[o] = 0
            if toggled > 0 or prev_state != new_state or not new_state:
                self.cooldown[o] = state_cooldown
            return toggled

        toggle_order, added = [], np.zeros(n, bool)
        applied = np.zeros(n, bool)
        for cands in ([i for i in range(n) if pending[i]], [i for i in order if desired[i]], vis_x, hid_x, order):
            for idx in cands:
                if not added[idx]:
                    toggle_order.append(idx)
                    added[idx] = True
        toggled_prims = 0
        for idx in toggle_order:
            if budget == 0 or toggled_prims >= budget:
                break
            want, current = bool(desired[idx]), bool(active[idx])
            if want == current:
                continue
            if self.cooldown[idx] > 0:
                if want:
                    pending[idx] = 1
                continue
            pend = int(self.counts[idx]) if want else int(self.counts[idx]) * int(current)
            if pend == 0:
                continue
            rem = budget - toggled_prims if budget > toggled_prims else 0
            if pend > rem:
                if want:
                    pending[idx] = 1
                continue
            t = set_object(idx, want)
            if t > 0:
                toggled_prims += min(t, rem)
                if want and not applied[idx]:
                    applied[idx] = True
                    pending[idx] = 0
                    self.desired_state[idx] = 1
                if not want:
                    X[idx] = f(0)
                    pending[idx] = 0
                    self.desired_state[idx] = 0
        if not active.any() and n > 0:
            fb = fallback if fallback < n else 0
            rem = budget - toggled_prims if budget > toggled_prims else 0
            if rem > 0:
                t = set_object(fb, True)
                toggled_prims += min(t, rem)
            self.desired_state[fb] = 1
            self.promoted[fb] = frame_no
        return active, toggled_prims


def _sanitize(v):
    fmax = np.finfo(np.float32).max
    v = np.float32(v)
    if np.isnan(v):
        return -fmax
    return min(max(v, -fmax), fmax)


def _libm_expf():
    import ctypes

    lm = ctypes.CDLL("libm.so.6")
    lm.expf.restype, lm.expf.argtypes = ctypes.c_float, [ctypes.c_float]
    return lambda x: np.float32(lm.expf(float(x)))


class EnvironmentOracle:
    """updateEnvironmentHitResidency (RendererResidency.cpp:4759-5155) and, with predictive=True,
    updatePredictiveResidency (:4397-4757), one object at a time, in numpy float32 (exp by libm
    expf, as the host build calls it), over the posterior of the same step."""

    def __init__(self, prim_counts, predictive=False):
        self.counts = np.asarray(prim_counts, np.int64)
        self.predictive = predictive
        self.cooldown = np.zeros(len(self.counts), np.int64)
        self.expf = _libm_expf()

    def decrement_cooldowns(self):
        self.cooldown = np.maximum(self.cooldown - 1, 0)

    def step(self, post, tests_last, score, visible, active, global_escape, target_fraction=0.25, min_active=16,
             max_toggles=20, camera_motion=0.0, memory_pressure=0.0, escape_threshold=0.4, high_escape=0.6,
             low_escape=0.3, state_cooldown=5):
        import math

        f = np.float32
        n = len(self.counts)
        active = np.asarray(active, bool).copy()
        vis = np.asarray(visible, bool)
        prim_count = int(self.counts.sum())

        def cl(v, lo=0.0, hi=1.0):
            return min(max(f(v), f(lo)), f(hi))

        motion, pressure = cl(camera_motion), cl(memory_pressure)
        thr = cl(f(escape_threshold) + f(0.03) * motion + f(0.08) * pressure, 0.12, 0.95)
        tf = cl(f(target_fraction) + f(0.08) * motion - f(0.10) * pressure, 0.12, 0.92 if self.predictive else 0.94)
        base = max(int(max_toggles), 1)
        budget = max(1, int(math.floor(base * (1.0 + 0.40 * float(motion) + 0.70 * float(pressure)) + 0.5)))
        importance = np.zeros(n, f)
        weighted = np.zeros(n, f)
        for o in range(n):
            prob = cl(post.probability[o])
            if not (int(tests_last[o]) > 0) and not active[o]:
                ex = max(f(post.exploration[o]), f(0))
                prior = f(1) - self.expf(-ex * f(0.5))
                if vis[o]:
                    prior = max(prior, f(1) - self.expf(-f(1) * f(0.5)))
                prior = cl(prior, 1.0e-4, 1.0)
                prob = max(prob, prior)
            importance[o] = prob
            sc = prob
            if self.predictive:
                hs = f(score[o])
                if self.counts[o] > 0:
                    hs = hs / f(self.counts[o])
                if hs <= 0 and (active[o] or vis[o]):
                    hs = f(1)
                sc = hs * prob
            w = sc * max(f(1), f(0)) * max(f(2) if vis[o] else f(0.05), f(0))
            weighted[o] = w if np.isfinite(w) else f(0)
        order = sorted(range(n), key=lambda o: (-weighted[o], -importance[o], o))
        min_act = min(prim_count, int(min_active))
        if min_act == 0 and prim_count > 0:
            min_act = 1
        target = 0
        if tf > 0 and prim_count > 0:
            target = min(int(math.ceil(tf * f(prim_count))), prim_count)
        floor = max(min_act, target)
        if not self.predictive:
            high = cl(high_escape)
            low = min(max(f(low_escape), f(0)), high)
            if f(global_escape) > high:
                floor = min(prim_count, int(f(floor) * f(1.5)))
            elif f(global_escape) < low:
                floor = max(min_act, int(f(floor) * f(0.8)))
        if floor == 0 and prim_count > 0:
            floor = 1
        desired = np.zeros(n, bool)
        count = 0
        wesc = f(0)
        for idx in order:
            c = int(self.counts[idx])
            if c == 0:
                continue
            avg = f(1) if count == 0 else wesc / f(count)
            if not (count < floor) and not (avg > thr):
                break
            desired[idx] = True
            count += c
            wesc = wesc + (f(1) - importance[idx]) * f(c)
        if count == 0 and prim_count > 0:
            for idx in order:
                if self.counts[idx] == 0:
                    continue
                desired[idx] = True
                break
        offscreen = int(sum(self.counts[o] for o in range(n) if active[o] and not vis[o]))
        max_budget = budget
        if offscreen > budget:
            max_budget = max(budget, (offscreen + 1) // 2)
        reserved = 0 if max_budget == 0 else max(1, max_budget // 4)
        general = max_budget - reserved if max_budget > reserved else 0
        total = max_budget + reserved
        toggled = 0

        def set_object(o, want):
            prev_state = bool(active[o])
            t = int(self.counts[o]) if want != prev_state else 0
            active[o] = want and self.counts[o] > 0
            if t > 0 or prev_state != bool(active[o]) or not active[o]:
                self.cooldown[o] = state_cooldown
            return t

        for idx in order:
            want, current = bool(desired[idx]), bool(active[idx])
            if want == current:
                continue
            bypass = current and not want and not vis[idx] and importance[idx] < thr
            if not bypass and self.cooldown[idx] > 0:
                continue
            if self.counts[idx] == 0:
                continue
            if toggled >= (total if bypass else general):
                continue
            t = set_object(idx, want)
            if t > 0:
                toggled = min(toggled + t, total)
        if not any(active[o] and self.counts[o] > 0 for o in range(n)):
            for idx in order:
                if self.counts[idx] == 0:
                    continue
                if set_object(idx, True) > 0:
                    break
        return active, toggled


def energy_static(sb):
    """Per-object summed primitive importance (primitiveImportance, Renderer.cpp:1482-1490) and
    emitted power times area, in primitive order, and the scene's total primitive importance,
    float32 as the library sums them."""
    f = np.float32
    g = sb.prims.reshape(-1, 28).astype(f)
    m = sb.materials.reshape(-1, 20).astype(f)
    t = g[:, 3].astype(np.int32)

    def lum(c):
        return (f(0.2126) * c[:, 0] + f(0.7152) * c[:, 1]) + f(0.0722) * c[:, 2]

    a = np.where((t == 1)[:, None], g[:, 4:7] - g[:, 0:3], g[:, 4:7]).astype(f)
    b = np.where((t == 1)[:, None], g[:, 8:11] - g[:, 0:3], g[:, 8:11]).astype(f)
    cx = a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1]
    cy = a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2]
    cz = a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]
    ln = np.sqrt((cx * cx + cy * cy) + cz * cz)
    area = np.where(t == 1, f(0.5) * ln, f(4.0) * ln).astype(f)
    area = np.where(t == 0, f(4.0) * f(np.pi) * g[:, 4] * g[:, 4], area).astype(f)
    emissive = m[:, 11] * lum(m[:, 8:11])
    op = m[:, 3]
    imp = (np.maximum(area, f(1e-4)) * (((emissive + lum(m[:, 0:3]) * op) + lum(m[:, 4:7]) * op) +
                                        (f(1) - op) * lum(m[:, 12:15]))).astype(f)
    emit = np.maximum(emissive * area, f(0)).astype(f)
    n = sb.object_count
    total, emit_o = np.zeros(n, f), np.zeros(n, f)
    inst = sb.instances
    for o in range(n):
        b0, c = int(inst["primitive_base"][o]), int(inst["primitive_count"][o])
        if c:
            total[o] = np.cumsum(np.maximum(imp[b0:b0 + c], f(0)), dtype=f)[-1]
            emit_o[o] = np.cumsum(emit[b0:b0 + c], dtype=f)[-1]
    return total, emit_o, np.cumsum(np.maximum(imp, f(0)), dtype=f)[-1]


class EnergyOracle:
    """updateEnergyImportance's object path without mesh groups (RendererResidency.cpp:1462-1860)
    in numpy float32, over the posterior, ray-hit score and screen coverage of the same step."""

    def __init__(self, sb):
        self.total, self.emit, self.prim_total = energy_static(sb)
        self.counts = sb.instances["primitive_count"].astype(np.int64)
        n = len(self.counts)
        self.hist = None
        self.cooldown = np.zeros(n, np.int64)
        self.last_toggle = np.zeros(n, np.int64)

    def decrement_cooldowns(self):
        self.cooldown = np.maximum(self.cooldown - 1, 0)

    def step(self, post, score, coverage, in_view, active, frame_no, width, height, target_fraction=0.88,
             min_active=16, max_toggles=32, camera_motion=0.0, memory_pressure=0.0, boost=1.75, smoothing=0.85,
             use_average=True, state_cooldown=5):
        import math

        f = np.float32
        n = len(self.counts)
        active = np.asarray(active, bool).copy()
        inv = np.asarray(in_view, bool)
        prim_count = int(self.counts.sum())

        def cl(v, lo=0.0, hi=1.0):
            return min(max(f(v), f(lo)), f(hi))

        motion, pressure = cl(camera_motion), cl(memory_pressure)
        tf = cl(f(target_fraction) + f(0.08) * motion - f(0.12) * pressure, 0.65, 0.97)
        budget = max(1, int(math.floor(max(int(max_toggles), 1) * (1.0 + 0.55 * float(motion) +
                                                                   0.35 * float(pressure)) + 0.5)))
        screen = f(width) * f(height)
        if screen <= 0:
            screen = f(1)
        bst = max(f(boost), f(1))
        apply_boost = bst > f(1.0001)
        max_emit = f(0)
        max_hit = f(0)
        imp = np.zeros(n, f)
        for o in range(n):
            max_emit = max(max_emit, self.emit[o])
            max_hit = max(max_hit, max(f(score[o]), f(0)))
            if apply_boost:
                frac = cl(f(coverage[o]) / screen)
                imp[o] = self.total[o] * (f(1) + (bst - f(1)) * frac)
            else:
                imp[o] = self.total[o]

        def norm(v, m):
            return f(0) if not (m > 0) else cl(f(v) / m)

        for o in range(n):
            hp = cl(post.probability[o])
            rh = norm(max(f(score[o]), f(0)), max_hit)
            en = norm(self.emit[o], max_emit)
            vw = f(1) if inv[o] else f(0)
            tr = ((((f(1) + f(0.90) * hp) + f(0.55) * rh) + f(0.40) * f(1)) + f(0.45) * vw) + f(0.90) * en
            imp[o] = imp[o] * tr
        hw = min(max(f(smoothing), f(0)), f(0.999))
        cw = f(1) - hw
        reset = self.hist is None
        if reset:
            self.hist = np.zeros(n, f)
        smoothed = np.zeros(n, f)
        for o in range(n):
            v = imp[o]
            if hw > 0:
                prev = imp[o] if reset else self.hist[o]
                v = prev * hw + imp[o] * cw
            self.hist[o] = v
            smoothed[o] = v
        boosted_total = f(0)
        if apply_boost:
            for v in smoothed:
                boosted_total = boosted_total + max(v, f(0))
        base = boosted_total if apply_boost else self.prim_total
        sel = np.zeros(n, f)
        total_sel = f(0)
        for o in range(n):
            v = smoothed[o]
            if use_average:
                if self.counts[o] == 0:
                    continue
                v = v / f(self.counts[o])
            sel[o] = v
            total_sel = total_sel + max(v, f(0))
        order = sorted(range(n), key=lambda o: (-_sanitize(sel[o]), o))
        min_act = min(prim_count, int(min_active))
        desired = np.zeros(n, bool)
        enabled = 0
        if self.prim_total <= 0:
            for idx in order:
                if self.counts[idx] == 0:
                    continue
                desired[idx] = True
                enabled += int(self.counts[idx])
                if enabled >= min_act:
                    break
        else:
            cum = f(0)
            target = (total_sel if total_sel > 0 else base) * tf
            for idx in order:
                c = int(self.counts[idx])
                if c == 0 and sel[idx] <= 0:
                    continue
                desired[idx] = True
                enabled += c
                cum = cum + max(sel[idx], f(0))
                if enabled >= min_act and cum >= target:
                    break
        if enabled < min_act:
            for idx in order:
                if desired[idx] or self.counts[idx] == 0:
                    continue
                desired[idx] = True
                enabled += int(self.counts[idx])
                if enabled >= min_act:
                    break
        toggled = 0

        def attempt(o, want):
            nonlocal toggled
            if want == bool(active[o]):
                return 0
            if self.cooldown[o] > 0:
                return 0
            last = self.last_toggle[o]
            if state_cooldown > 0 and last != 0 and frame_no >= last and frame_no - last < state_cooldown:
                return 0
            if self.counts[o] == 0:
                return 0
            if toggled >= budget:
                return 0
            prev = bool(active[o])
            t = int(self.counts[o])
            active[o] = want
            if prev != bool(active[o]):
                self.last_toggle[o] = frame_no
            self.cooldown[o] = state_cooldown
            toggled = min(toggled + t, budget)
            return t

        for o in range(n):
            attempt(o, bool(desired[o]))
        if not any(active[o] and self.counts[o] > 0 for o in range(n)):
            for idx in order:
                if self.counts[idx] == 0:
                    continue
                if attempt(idx, True) > 0:
                    break
        return active, toggled
