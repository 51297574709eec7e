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


def select(keys, visible, nbytes, budget, reserve, min_active, current, max_toggles=0, always=False):
    n = keys.shape[0]
    k = np.where(np.isfinite(keys), keys, 0.0).astype(np.float32)
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
