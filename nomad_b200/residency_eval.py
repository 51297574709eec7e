"""Learned-residency workload: dataset recording, on-device training and the policy comparison.

Workload (the learned-residency configuration): a city of 2,048 objects (~6M triangles), a
300-frame seeded Catmull-Rom camera path, a geometry budget of 40% of all object bytes. Every
frame renders the view with the current resident set (per-object hit counting on), then runs
one residency step. The image judge is the same frame rendered with every object resident
(a second context, same Philox streams), compared in HDR:
rel-MSE = mean((I - I_AR)^2) / mean(I_AR^2), averaged over the frames whose reference is not
black (also reported: its median, and the energy-weighted sum(num) / sum(den) over the path, which
near-black reference frames cannot dominate).

The learned scorer is trained on the device on hit counts recorded along seeded training camera
paths rendered with every object resident: features of frame f, target log1p(hits of frame
f+1). To cover what the policy sees once it evicts objects (no hits, decaying history), a copy
of every sample has its hit-history features replaced by the evicted pattern.
"""
from __future__ import annotations

import time

import numpy as np

from . import native as nat

HIST_FEATURES = list(range(3, 12)) + [19, 20]


def catmull_rom(points: np.ndarray, n: int) -> np.ndarray:
    """n positions along a uniform Catmull-Rom spline through points (k x 3)."""
    p = np.concatenate([points[:1], points, points[-1:]])
    segs = len(points) - 1
    out = []
    for i in range(n):
        u = i * segs / max(n - 1, 1)
        s = min(int(u), segs - 1)
        t = u - s
        p0, p1, p2, p3 = p[s], p[s + 1], p[s + 2], p[s + 3]
        t2, t3 = t * t, t * t * t
        out.append(0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t2
                          + (-p0 + 3 * p1 - 3 * p2 + p3) * t3))
    return np.asarray(out, np.float32)


def camera_path(seed: int, frames: int, extent_x: float, extent_z: float, controls: int = 8):
    """Seeded path over the city: positions at 15-90 m height, looking 60 m ahead and down."""
    rng = np.random.default_rng(seed)
    ctrl = np.stack([rng.uniform(-0.45, 0.45, controls) * extent_x, rng.uniform(15, 90, controls),
                     rng.uniform(-0.45, 0.45, controls) * extent_z], 1)
    pos = catmull_rom(ctrl, frames + 1)
    views = []
    for i in range(frames):
        d = pos[i + 1] - pos[i]
        d[1] = 0.0
        n = np.linalg.norm(d)
        d = d / n if n > 1e-4 else np.array([0.0, 0.0, 1.0], np.float32)
        look = pos[i] + d * 60.0 - np.array([0.0, 25.0, 0.0], np.float32)
        views.append((pos[i], look))
    return views


def make_view(pos, look, width, height, spp, depth, seed, frame):
    return nat.view_pinhole(pos, look, width=width, height=height, spp=spp, max_depth=depth,
                            seed=seed, frame=frame)


class Workload:
    def __init__(self, seed=17, grid=64, grid_z=32, size_m=2000.0, target_tris=6_000_000,
                 width=640, height=360, spp=2, depth=2, frames=300, budget_fraction=0.4):
        t0 = time.perf_counter()
        self.scene = nat.synth_city(seed, grid=grid, grid_z=grid_z, size_m=size_m,
                                    target_tris=target_tris, emissive_quads=64)
        self.sb = nat.SceneBVH(self.scene)
        self.extent = (size_m, size_m * grid_z / grid)
        self.width, self.height, self.spp, self.depth = width, height, spp, depth
        self.frames = frames
        self.seed = seed
        self.budget_fraction = budget_fraction
        self.setup_s = time.perf_counter() - t0

    def tune(self, ctx, judge=None):
        """Autotunes the traversal on the primary rays of a path's first view; the judge context
        gets the same configuration. Returns the configuration's name."""
        from .rays import Camera

        pos, look = camera_path(1, 2, *self.extent)[0]
        cam = Camera(tuple(float(x) for x in pos), tuple(float(x) for x in look), width=self.width,
                     height=self.height)
        res = ctx.autotune_sweep(cam.primary_rays(self.spp, seed=3), repeats=2)
        if judge is not None:
            judge.set_traversal(**res["best"])
        return res["best_name"]

    def context(self, device=0):
        c = nat.Context(device)
        c.upload(self.sb)
        return c

    def views(self, path_seed, frames):
        return [make_view(p, l, self.width, self.height, self.spp, self.depth, self.seed, f)
                for f, (p, l) in enumerate(camera_path(path_seed, frames, *self.extent))]

    # ---- training data ---------------------------------------------------------------------
    def record(self, ctx, paths=200, frames_per_path=8, first_path_seed=1000):
        """(features, targets) under AlwaysResident along seeded training paths."""
        prm = nat.ResidencyParams.make(nat.POLICY_ALWAYS)
        feats, targs = [], []
        for p in range(paths):
            views = self.views(first_path_seed + p, frames_per_path + 1)
            prev = None
            for f, v in enumerate(views):
                ctx.reset_object_hits()
                ctx.render(v, count_hits=True)
                hits = ctx.object_hits().astype(np.float32)
                if prev is not None:
                    feats.append(prev)
                    targs.append(np.log1p(hits))
                ctx.residency_step(prm, v)
                prev = ctx.residency_last()[0].copy()
        x = np.concatenate(feats)
        t = np.concatenate(targs).astype(np.float32)
        # evicted-pattern copies: no recent hits, no score, long time since the last hit
        xe = x.copy()
        xe[:, HIST_FEATURES] = 0.0
        xe[:, 19] = np.log1p(255.0)
        xe[:, 18] = 0.0
        return np.concatenate([x, xe]), np.concatenate([t, t])

    def train(self, ctx, x, t, steps=1500, batch=4096, lr=2e-3, seed=5):
        ctx.mlp_init(seed)
        return ctx.mlp_train(x, t, steps=steps, batch=batch, lr=lr, weight_decay=1e-4, seed=seed)

    # ---- evaluation ------------------------------------------------------------------------
    def evaluate(self, ctx, judge, policy, path_seed=1, frames=None, warm=5, budget_fraction=None, prm=None):
        """Runs the camera path with one policy; returns per-frame rel-MSE and timings."""
        import torch

        frames = frames or self.frames
        views = self.views(path_seed, frames)
        nbytes = ctx.object_bytes()
        budget = int((budget_fraction or self.budget_fraction) * nbytes.sum())
        if prm is None:
            prm = nat.ResidencyParams.make(policy, budget_bytes=budget if policy != nat.POLICY_ALWAYS else 0,
                                           camera_motion=0.3, min_active=0)
        # start from everything resident, as the reference's AlwaysResident warm-up does
        ctx.residency_step(nat.ResidencyParams.make(nat.POLICY_ALWAYS), views[0])
        ctx.reset_object_hits()
        npix = self.width * self.height
        d_img = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
        d_ref = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
        mse, ms, resident_bytes = [], [], []
        sum_num = sum_den = 0.0
        for f, v in enumerate(views):
            judge.render_dev(v, d_ref.data_ptr())
            judge.sync()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ctx.render_dev(v, d_img.data_ptr(), count_hits=True)
            ctx.residency_step(prm, v, toggles=prm.policy in (nat.POLICY_RAYHIT_PRIM, nat.POLICY_DISTANCE_LOD,
                                                             nat.POLICY_SCREEN_SPACE))
            ctx.sync()
            dt = time.perf_counter() - t0
            num = torch.mean((d_img - d_ref) ** 2).item()
            den = torch.mean(d_ref ** 2).item()
            if f >= warm:
                if den > 0:  # a black reference frame (camera inside geometry) has no relative error
                    mse.append(num / den)
                sum_num += num
                sum_den += den
                ms.append(dt * 1e3)
                flags = ctx.residency_flags().astype(bool)
                resident_bytes.append(int(nbytes[flags].sum()))
        return {"rel_mse": float(np.mean(mse)), "rel_mse_p50": float(np.median(mse)),
                "rel_mse_energy": sum_num / sum_den if sum_den > 0 else None,
                "ms_per_frame": float(np.mean(ms)),
                "ms_per_frame_p50": float(np.median(ms)),
                "resident_fraction": float(np.mean(resident_bytes) / nbytes.sum()),
                "frames": len(mse)}


    def evaluate_paged(self, ctx, judge, policy, path_seed=1, frames=None, warm=5, pool_slack=1.25):
        """The same run with geometry paging: a third context whose BLAS nodes (of the tuned
        traversal width) and triangle records live in a device pool of pool_slack x the budget's
        share of the paged bytes, streamed in by nomad_paging_update after every residency step
        (at most 32 onloads per frame). ms/frame includes the update; rel-MSE includes the frames
        where wanted objects are still streaming."""
        import torch

        frames = frames or self.frames
        views = self.views(path_seed, frames)
        trav = ctx.traversal()
        probe = self.context()
        probe.set_traversal(**trav)
        probe.paging_enable(1 << 50, width=trav["width"])
        full = probe.paging_stats()["full_bytes"]
        probe.close()
        pc = self.context()
        try:
            pc.set_traversal(**trav)
            pc.mlp_set(ctx.mlp_get())
            pool = int(min(full, full * self.budget_fraction * pool_slack))
            pc.paging_enable(pool, width=trav["width"])
            nbytes = pc.object_bytes()
            budget = int(self.budget_fraction * nbytes.sum())
            prm = nat.ResidencyParams.make(policy, budget_bytes=budget, camera_motion=0.3, min_active=0)
            pc.reset_object_hits()
            npix = self.width * self.height
            d_img = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
            d_ref = torch.empty(npix * 3, dtype=torch.float32, device="cuda")
            mse, ms, streamed, onl = [], [], [], []
            sum_num = sum_den = 0.0
            prev = pc.paging_stats()
            for f, v in enumerate(views):
                judge.render_dev(v, d_ref.data_ptr())
                judge.sync()
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                pc.render_dev(v, d_img.data_ptr(), count_hits=True)
                pc.residency_step(prm, v, toggles=False)
                pc.paging_update()
                pc.sync()
                dt = time.perf_counter() - t0
                num = torch.mean((d_img - d_ref) ** 2).item()
                den = torch.mean(d_ref ** 2).item()
                st = pc.paging_stats()
                if f >= warm:
                    mse.append(num / den if den > 0 else None)
                    sum_num += num
                    sum_den += den
                    ms.append(dt * 1e3)
                    streamed.append(st["bytes_streamed"] - prev["bytes_streamed"])
                    onl.append(st["onloads"] - prev["onloads"])
                prev = st
            st = pc.paging_stats()
            late = [m for m in mse[max(0, 40 - warm):] if m is not None]
            mse = [m for m in mse if m is not None]
            return {"rel_mse": float(np.mean(mse)), "rel_mse_p50": float(np.median(mse)),
                    "rel_mse_energy": sum_num / sum_den if sum_den > 0 else None,
                    "rel_mse_from_frame_40": float(np.mean(late)) if late else None,
                    "ms_per_frame": float(np.mean(ms)),
                    "ms_per_frame_p50": float(np.median(ms)), "frames": len(mse),
                    "pool_bytes": st["pool_bytes"], "full_paged_bytes": st["full_bytes"],
                    "mean_streamed_bytes_per_frame": float(np.mean(streamed)),
                    "mean_onloads_per_frame": float(np.mean(onl)), "max_onloads_per_frame": int(np.max(onl)),
                    "denied": st["denied"], "deferred": st["deferred"], "evictions": st["evictions"],
                    "relinks_from_cache": st["relinks"], "resident_objects_end": st["resident"],
                    "cached_objects_end": st["cached"]}
        finally:
            pc.close()


def run(paths=200, frames_per_path=8, steps=1500, frames=300, log=print):
    """Full comparison; returns a dict for the bench line."""
    t0 = time.perf_counter()
    w = Workload(frames=frames)
    log(f"residency workload: {w.sb.prim_count} prims, {w.sb.object_count} objects, set-up {w.setup_s:.1f}s")
    ctx = w.context()
    judge = w.context()
    traversal = w.tune(ctx, judge)
    log(f"traversal: {traversal}")
    t1 = time.perf_counter()
    x, t = w.record(ctx, paths=paths, frames_per_path=frames_per_path)
    t2 = time.perf_counter()
    loss = w.train(ctx, x, t, steps=steps)
    t3 = time.perf_counter()
    log(f"recorded {x.shape[0]} samples in {t2 - t1:.1f}s, trained {steps} steps in {t3 - t2:.1f}s, "
        f"loss {loss[:10].mean():.4f} -> {loss[-50:].mean():.4f}")
    out = {"workload": f"city {w.sb.object_count} objects / {w.sb.prim_count} prims, {frames}-frame path, "
                       f"{w.width}x{w.height} x {w.spp} spp, {w.depth} bounces, budget "
                       f"{int(100 * w.budget_fraction)}% of geometry bytes",
           "traversal": traversal,
           "train": {"samples": int(x.shape[0]), "steps": steps, "loss_first": float(loss[:10].mean()),
                     "loss_last": float(loss[-50:].mean()), "record_s": t2 - t1, "train_s": t3 - t2}}
    for name, pol in (("always_resident", nat.POLICY_ALWAYS), ("ray_hit_budget", nat.POLICY_RAYHIT_BUDGET),
                      ("learned", nat.POLICY_LEARNED)):
        out[name] = w.evaluate(ctx, judge, pol, frames=frames)
        log(f"{name}: {out[name]}")
    for name, pol in (("ray_hit_budget_paged", nat.POLICY_RAYHIT_BUDGET), ("learned_paged", nat.POLICY_LEARNED)):
        try:
            out[name] = w.evaluate_paged(ctx, judge, pol, frames=frames)
        except nat.NomadError as exc:  # a traversal width the paging cannot hold
            out[name] = {"error": str(exc)}
        log(f"{name}: {out[name]}")
    # The reference's host-side heuristics switch objects and primitives through the residency
    # interface, which a later device step does not undo: each runs on a fresh context with the
    # tuned traversal, so no leg sees another's toggles.
    def host_leg(policy, prm, n_frames):
        pc = w.context()
        try:
            pc.set_traversal(**ctx.traversal())
            return w.evaluate(pc, judge, policy, frames=n_frames, prm=prm)
        finally:
            pc.close()

    # The reference's own per-primitive ray-hit policy (host, per primitive, its defaults: 54 %
    # of the primitives, 16 toggles a frame, cooldowns), on a shorter path.
    out["ray_hit_per_primitive_reference"] = host_leg(
        nat.POLICY_RAYHIT_PRIM,
        nat.ResidencyParams.make(nat.POLICY_RAYHIT_PRIM, max_toggles=16, camera_motion=0.3, min_active=16),
        min(frames, 100))
    log(f"ray_hit_per_primitive_reference: {out['ray_hit_per_primitive_reference']}")
    # The reference's DistanceLOD heuristic with its defaults (225 / 275 m, 5 / 12 degrees, 24
    # toggles a frame), host-side per object.
    out["distance_lod_reference"] = host_leg(
        nat.POLICY_DISTANCE_LOD,
        nat.ResidencyParams.make(nat.POLICY_DISTANCE_LOD, max_toggles=24, camera_motion=0.3), frames)
    log(f"distance_lod_reference: {out['distance_lod_reference']}")
    # The reference's ScreenSpaceFootprint heuristic with its defaults (68 % of the screen, 32 px,
    # 14 primitive toggles a frame), one mesh group per object.
    out["screen_space_reference"] = host_leg(
        nat.POLICY_SCREEN_SPACE,
        nat.ResidencyParams.make(nat.POLICY_SCREEN_SPACE, max_toggles=14, camera_motion=0.3, min_active=16,
                                 target_fraction=0.68, min_pixel_coverage=32.0), frames)
    log(f"screen_space_reference: {out['screen_space_reference']}")
    # The learned policy at smaller budgets: the smallest one whose rel-MSE is within 5 % of the
    # ray-hit policy's at the full budget, and its ms/frame.
    sweep = {}
    for frac in (0.1, 0.15, 0.2, 0.25, 0.3):
        sweep[f"{frac:.2f}"] = w.evaluate(ctx, judge, nat.POLICY_LEARNED, frames=frames, budget_fraction=frac)
    out["learned_budget_sweep"] = sweep
    target = 1.05 * out["ray_hit_budget"]["rel_mse"]
    ok = [k for k, v in sorted(sweep.items()) if v["rel_mse"] <= target]
    out["learned_matching_rayhit"] = ({"budget_fraction": float(ok[0]), **sweep[ok[0]],
                                       "ray_hit_ms_per_frame": out["ray_hit_budget"]["ms_per_frame"]}
                                      if ok else None)
    log(f"learned budget sweep: { {k: (v['rel_mse'], v['ms_per_frame']) for k, v in sweep.items()} }")
    rh, le = out["ray_hit_budget"]["rel_mse"], out["learned"]["rel_mse"]
    out["learned_vs_rayhit_rel_mse_ratio"] = le / rh if rh > 0 else None
    out["total_s"] = time.perf_counter() - t0
    ctx.close()
    judge.close()
    return out


if __name__ == "__main__":
    import json
    import sys

    args = dict(a.split("=") for a in sys.argv[1:])
    res = run(paths=int(args.get("paths", 200)), frames_per_path=int(args.get("fpp", 8)),
              steps=int(args.get("steps", 1500)), frames=int(args.get("frames", 300)))
    print(json.dumps(res))
