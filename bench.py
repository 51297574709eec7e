#!/usr/bin/env python
"""Closest-hit throughput on the 2.5M-triangle synthetic city at 1080p.

One step = the closest-hit pass over one frame's ray batch of the city workload:
1920x1080 pixels x 4 jittered primary rays (8,294,400 rays) followed by one cosine-weighted
diffuse bounce ray for every primary hit, each batch one launch of the traversal kernel.
`value` is Mrays/s with the rays already resident in HBM; `e2e` is the same metric through the
C ABI with host (pinned) ray and hit buffers, the copies inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Multi-GPU: one process per GPU (torchrun); every rank traces its own replica of the frame
(views are independent; no collective on the data path) and rank 0 reports the aggregate.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time
import types

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 2
WIDTH, HEIGHT, SPP = 1920, 1080, 4
METRIC = "closest-hit Mrays/s (city 1080p x4spp + bounce)"
CONFIG = {
    "workload": "synthetic city: 1,024 objects, ~2.5M FP32 triangles (lognormal per-object "
                "counts, median 1k, max 200k), 64 emissive quads; 1920x1080 x 4 spp jittered "
                "primary rays + 1 diffuse bounce per primary hit; closest-hit",
    "scene_seed": SEED, "width": WIDTH, "height": HEIGHT, "spp": SPP,
    "l2": "inputs larger than L2 (rays 265 MB + 160 MB, traversal layout 233 MB)",
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "20"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.time(), line.strip()))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t_begin=None, t_end=None):
        """Median SM clock and active throttle reasons over the samples taken inside
        [t_begin, t_end] (host wall time; all samples when no window is given, the first
        sample after t_begin when the window is shorter than the sampling period)."""
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        rows = self.lines
        if t_begin is not None:
            inside = [r for r in rows if t_begin - 0.02 <= r[0] <= t_end + 0.02]
            if not inside:
                inside = [r for r in rows if r[0] >= t_begin][:1]
            rows = inside
        for _, ln in rows:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


TRAFFIC_PROFILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles",
                               "k_trace_dram_profile_case_bvh4_persist_mb10.md")


def measured_traffic(rays):
    """Per-launch DRAM bytes (read + write) of the primary and bounce launches: the DRAM bytes per
    ray that one ncu capture of the two k_trace launches of `--profile-case` measured (recorded in
    the profile summary), times this step's rays per launch (`rays`: {"primary": n, "bounce": n}).
    None when the summary is absent."""
    try:
        vals = {}
        with open(TRAFFIC_PROFILE) as f:
            for line in f:
                for key in ("primary", "bounce"):
                    tag = f"traffic_{key}_bytes_per_ray:"
                    if line.strip().startswith(tag):
                        vals[key] = float(line.strip()[len(tag):].strip().strip("`"))
        if len(vals) != 2:
            return None
        return {k: int(round(vals[k] * rays[k])) for k in vals}
    except OSError:
        return None


def build_workload(nb, spp=SPP):
    scene = nb.synth_city(seed=SEED)
    sb = nb.SceneBVH(scene)
    cam = nb.city_camera(WIDTH, HEIGHT)
    primary = cam.primary_rays(spp, seed=SEED + 10)
    return scene, sb, primary


def cpu_leg(sb, rays, budget_s=12.0, use_reference=False):
    """Times the CPU traversal on the host cores over a bounded sample of the workload."""
    cores = len(os.sched_getaffinity(0))
    if use_reference:
        from oracle import reference as ref
        if not ref.available():
            use_reference = False
    from oracle import oracle as orc
    os_ = orc.OracleScene(sb)
    rng = np.random.default_rng(123)
    sample = rays[rng.permutation(rays.shape[0])]
    done, t0 = 0, time.perf_counter()
    chunk = 200_000
    # Cycle through the shuffled batch until the time budget is spent.
    while time.perf_counter() - t0 < budget_s and done < 20 * sample.shape[0]:
        off = done % sample.shape[0]
        part = sample[off:off + chunk]
        if use_reference:
            ref.closest(sb, part, threads=cores)
        else:
            os_.closest(part, orc.MODE_REFERENCE_ORDER, threads=cores)
        done += part.shape[0]
    dt = time.perf_counter() - t0
    out = {"value": done / dt / 1e6, "unit": "Mrays/s", "cores": cores,
           "kind": "reference" if use_reference else "port",
           "sample": f"{done} rays drawn uniformly from the workload's primary+bounce batch "
                     f"({dt:.1f} s of CPU work, {cores} threads)"}
    if not use_reference:
        out.update(cpu_extra(os_, orc, sb, sample, cores))
    return out


def cpu_extra(os_, orc, sb, sample, cores, budget_s=4.0):
    """The scalar port's any-hit rate over the same rays (tmax as given), and its path-traced
    ms per C2 frame (1920x1080 x 4 spp, 3 bounces, NEE) extrapolated from a seeded sample of
    pixels rendered in full (all samples and bounces of each)."""
    done, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and done < sample.shape[0]:
        part = sample[done:done + 200_000]
        os_.any(part, orc.MODE_REFERENCE_ORDER, threads=cores)
        done += part.shape[0]
    dt_any = time.perf_counter() - t0
    import nomad_b200 as nb

    v = nb.view_pinhole((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), width=WIDTH, height=HEIGHT, spp=SPP,
                        max_depth=3, seed=SEED)
    px = np.random.default_rng(321).permutation(WIDTH * HEIGHT).astype(np.uint64)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and n < px.size:
        orc.render(os_, sb.materials, v, pixels=px[n:n + 1024], threads=cores)
        n += 1024
    dt_pt = time.perf_counter() - t0
    return {"any_hit_mrays_s": done / dt_any / 1e6,
            "path_traced_ms_per_frame": dt_pt / n * WIDTH * HEIGHT * 1e3,
            "path_traced_sample": f"{n} seeded pixels of the C2 frame, every sample and bounce "
                                  f"({dt_pt:.1f} s, {cores} threads), scaled to {WIDTH * HEIGHT} pixels"}


def frame_leg(nb, ctx, sb, frames=3):
    """Path-traced city frame (1920x1080 x 4 spp, 3 bounces, NEE): ms/frame and ray rates."""
    import torch

    v = nb.view_pinhole((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), width=WIDTH, height=HEIGHT, spp=SPP,
                        max_depth=3, seed=SEED)
    out = torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32, device="cuda")
    ctx.render_dev(v, out.data_ptr())
    ctx.sync()
    ctx.reset_render_stats()
    t0 = time.perf_counter()
    for f in range(frames):
        v["frame"] = f
        ctx.render_dev(v, out.data_ptr())
    ctx.sync()
    dt = (time.perf_counter() - t0) / frames
    st = ctx.render_stats() / frames
    return {"config": "city 1920x1080 x 4 spp, 3 bounces, one-sample NEE", "ms_per_frame": dt * 1e3,
            "closest_rays_per_frame": int(st[0]), "shadow_rays_per_frame": int(st[2]),
            "mrays_per_s_incl_shadow": (st[0] + st[2]) / dt / 1e6}


def split_frame_leg(nb, ctx, world, frames=5):
    """The path-traced city frame of frame_leg split over the ranks by row bands
    (nomad_b200.split_frame: each rank renders its rows as a tile, the bands are all-gathered on
    the device). Every rank runs it, with the same collectives in the same order; ms/frame is the
    slowest rank's time from its first band's launch to the gathered frame."""
    import torch
    import torch.distributed as dist

    from nomad_b200.split_frame import render_split, row_bands

    v = nb.view_pinhole((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), width=WIDTH, height=HEIGHT, spp=SPP,
                        max_depth=3, seed=SEED)
    render_split(ctx, v)  # captures the band's frame graph
    torch.cuda.synchronize()
    dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for f in range(frames):
        v["frame"] = f
        img = render_split(ctx, v)[0]
    e1.record()
    e1.synchronize()
    ms = ranks_max(e0.elapsed_time(e1) / frames, world)
    return {"config": f"city {WIDTH}x{HEIGHT} x {SPP} spp, 3 bounces, one-sample NEE, rows split over {world} ranks",
            "ms_per_frame": ms, "rows_per_rank": [b[1] for b in row_bands(HEIGHT, world)],
            "frame_shape": list(img.shape), "frames": frames}


def multiview_views(nb, n=16, seed=404):
    rng = np.random.default_rng(seed)
    views = []
    for i in range(n):
        w = int(rng.integers(256, 1921))
        h = int(np.clip(rng.integers(256, 1081), 256, 1080))
        ang = rng.uniform(0, 2 * np.pi)
        pos = (float(450 * np.cos(ang)), float(rng.uniform(40, 250)), float(450 * np.sin(ang)))
        views.append(nb.view_pinhole(pos, (0.0, 0.0, 0.0), width=w, height=h, spp=int(rng.integers(1, 17)),
                                     max_depth=2, seed=SEED + i))
    return np.concatenate(views)


def multiview_leg(nb, ctx, frames=3):
    """16 views of the city at seeded uneven sizes (256..1920 x 256..1080) and spp (1..16),
    2 bounces, all paths in one batched launch sequence per frame."""
    import torch

    views = multiview_views(nb)
    px = int((views["width"].astype(np.int64) * views["height"]).sum())
    paths = int((views["width"].astype(np.int64) * views["height"] * views["spp"]).sum())
    out = torch.empty(px * 3, dtype=torch.float32, device="cuda")
    timings = {}
    for mode in ("direct", "graph"):
        graph = mode == "graph"
        ctx.render_dev(views, out.data_ptr(), graph=graph)  # warm-up (captures the graph)
        ctx.sync()
        g0 = ctx.frame_graph_stats()
        ctx.reset_render_stats()
        t0 = time.perf_counter()
        for f in range(frames):
            views["frame"] = f
            ctx.render_dev(views, out.data_ptr(), graph=graph)
        ctx.sync()
        timings[mode] = (time.perf_counter() - t0) / frames
        st = ctx.render_stats() / frames
        g1 = ctx.frame_graph_stats()
    dt = timings["graph"]
    return {"views": int(views.shape[0]), "pixels": px, "paths": paths, "ms_per_frame": dt * 1e3,
            "ms_per_frame_direct_launches": timings["direct"] * 1e3,
            "graph_replays_timed": g1["launches"] - g0["launches"],
            "graph_captures_timed": g1["captures"] - g0["captures"],
            "mpaths_per_s": paths / dt / 1e6, "mrays_per_s_incl_shadow": (st[0] + st[2]) / dt / 1e6}


def restir_leg(nb, ctx, frames=8):
    """ReSTIR DI on the city with 4,096 emissive triangles (lognormal power, sigma 1.5): per frame
    of an 8-frame spline move, rel-MSE of 1-spp direct lighting against a 1024-spp reference
    (pixel centres, 480x270), for ReSTIR (32 candidates, 1 temporal + 3 spatial within 30 px,
    M-cap 20) and for one-sample NEE; and ReSTIR ms/frame at 1920x1080 x 1 spp."""
    import torch

    from nomad_b200.residency_eval import catmull_rom

    scene = nb.synth_city(seed=SEED, emissive_tris=4096, emissive_sigma=1.5)
    sb2 = nb.SceneBVH(scene)
    c2 = nb.Context(0)
    c3 = nb.Context(0)  # the reference's own ReSTIR, with its own reservoir history
    try:
        c2.upload(sb2)
        c2.set_restir(candidates=32, temporal=True, spatial=3, radius_px=30.0, m_cap=20.0)
        c3.upload(sb2)
        c3.set_restir(candidates=32, temporal=True, reference_mode=True)
        rng = np.random.default_rng(SEED + 3)
        ctrl = np.stack([rng.uniform(-150, 150, 5), rng.uniform(120, 220, 5), rng.uniform(-650, -500, 5)], 1)
        path = catmull_rom(ctrl, frames)
        W, H = 480, 270
        errs = {"restir": [], "nee": [], "restir_reference_mode": []}
        for f in range(frames):
            pos = tuple(float(x) for x in path[f])
            ref = c2.render(nb.view_pinhole(pos, (0.0, 0.0, 60.0), width=W, height=H, spp=1024, max_depth=1,
                                            seed=9000 + f, flags=nb.VIEW_CENTER))[0]
            den = float((ref.astype(np.float64) ** 2).mean())
            for name, cx, fl in (("restir", c2, nb.VIEW_RESTIR), ("nee", c2, 0),
                                 ("restir_reference_mode", c3, nb.VIEW_RESTIR)):
                img = cx.render(nb.view_pinhole(pos, (0.0, 0.0, 60.0), width=W, height=H, spp=1, max_depth=1,
                                                seed=7, frame=f, flags=fl | nb.VIEW_CENTER))[0]
                errs[name].append(float(((img.astype(np.float64) - ref) ** 2).mean() / den))
        out = torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32, device="cuda")
        v = nb.view_pinhole((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), width=WIDTH, height=HEIGHT, spp=1,
                            max_depth=1, seed=SEED, flags=nb.VIEW_RESTIR)
        c2.render_dev(v, out.data_ptr())
        c2.sync()
        t0 = time.perf_counter()
        for f in range(4):
            v["frame"] = f + 1
            c2.render_dev(v, out.data_ptr())
        c2.sync()
        ms = (time.perf_counter() - t0) / 4 * 1e3
        c3.render_dev(v, out.data_ptr())
        c3.sync()
        t0 = time.perf_counter()
        for f in range(4):
            v["frame"] = f + 1
            c3.render_dev(v, out.data_ptr())
        c3.sync()
        ms_ref = (time.perf_counter() - t0) / 4 * 1e3
        return {"config": "city + 4,096 emissive tris, 8-frame spline, 480x270 error / 1080p timing",
                "rel_mse_per_frame": errs, "rel_mse_mean": {k: float(np.mean(v)) for k, v in errs.items()},
                "restir_ms_per_frame_1080p_1spp": ms,
                "restir_reference_mode_ms_per_frame_1080p_1spp": ms_ref}
    finally:
        c2.close()
        c3.close()


def compaction_leg(nb, sb, primary, steps=10):
    """Residency compaction on the device (nomad_scenebvh_compact_gpu) of the 2.5M-triangle city
    under a seeded 40 % object mask: ms per compaction (CUDA events, inputs larger than L2), the
    bytes it must move, and closest-hit Mrays/s of the primary rays on the compacted scene next
    to the same scene with the mask applied to the full arrays."""
    import torch

    rng = np.random.default_rng(SEED + 40)
    objs = rng.random(sb.object_count) < 0.4
    active = objs[sb.prim_object].astype(np.uint8)
    stream = torch.cuda.Stream()
    prev = torch.cuda.current_stream()
    torch.cuda.set_stream(stream)  # compaction, traces and events all on one stream
    comp = nb.native.Compactor(sb)
    act_dev = torch.from_numpy(active).cuda()
    for _ in range(3):
        comp.run(act_dev)
    torch.cuda.synchronize()
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record()
    for _ in range(steps):
        comp.run(act_dev)
    t1.record()
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1) / steps
    c = comp.result()
    n, nodes, p = sb.prim_count, sb.bvh_node_count, c["prim_count"]
    # read: index + flag per primitive, node words, the active primitives' records; written: the
    # compact primitive, material, index, remap and the global map, the kept nodes
    moved = n * (4 + 1 + 4) + nodes * 32 + p * (112 + 80) * 2 + p * 8 + n * 4 + c["bvh_node_count"] * 32
    cs = types.SimpleNamespace(
        bvh_nodes=c["bvh_nodes"], bvh_node_count=c["bvh_node_count"], tlas_nodes=sb.tlas_nodes,
        tlas_node_count=sb.tlas_node_count, prims=c["prims"], materials=c["materials"],
        prim_indices=c["prim_indices"], prim_count=p, instances=c["instances"], object_count=sb.object_count)
    rays = np.ascontiguousarray(primary)
    d_rays = torch.from_numpy(rays.view(np.uint8)).cuda()
    d_hits = torch.empty(rays.shape[0] * 20, dtype=torch.uint8, device="cuda")
    rates = {}
    for name in ("masked", "compacted"):
        ctx = nb.Context()
        try:
            if name == "masked":
                ctx.upload(sb)
                for o in np.nonzero(~objs)[0]:
                    ctx.set_object_active(int(o), False)
                ctx.flush()
            else:
                ctx.upload(cs)
            ctx.set_stream(stream.cuda_stream)
            for _ in range(3):
                ctx.trace_closest_dev(d_rays.data_ptr(), rays.shape[0], d_hits.data_ptr())
            torch.cuda.synchronize()
            t0.record()
            for _ in range(steps):
                ctx.trace_closest_dev(d_rays.data_ptr(), rays.shape[0], d_hits.data_ptr())
            t1.record()
            torch.cuda.synchronize()
            rates[name] = rays.shape[0] * steps / (t0.elapsed_time(t1) / 1e3) / 1e6
        finally:
            ctx.close()
    torch.cuda.set_stream(prev)
    return {"ms": ms, "active_objects": int(objs.sum()), "objects": int(sb.object_count),
            "resident_prims": p, "prims": int(n), "compact_nodes": c["bvh_node_count"], "nodes": int(nodes),
            "algorithmic_bytes": int(moved), "achieved_gbs": moved / (ms / 1e3) / 1e9,
            "geometry_bytes": {"full": int(n * 196 + nodes * 32), "compacted": int(p * 196 + c["bvh_node_count"] * 32)},
            "closest_mrays_s": rates}


def residency_leg():
    from nomad_b200 import residency_eval

    return residency_eval.run(log=log)


def run_profile_case(args):
    """The bench workload at a quarter of the pixels, for ncu captures: the city, 960x540 x 4
    jittered primary rays (2,073,600, the bench's density of rays per pixel and seeds) and one
    diffuse bounce per primary hit, all on the device. k_trace launches: one to make the
    primary hits the bounces start from, then three iterations of (primary launch, bounce
    launch) with the chosen variant; the hits must agree across iterations. Capturing
    `-k regex:k_trace -s 3 -c 2` takes the second iteration's primary and bounce launches."""
    import torch

    import nomad_b200 as nb

    scene = nb.synth_city(seed=SEED)
    sb = nb.SceneBVH(scene)
    ctx = nb.Context(0)
    ctx.upload(sb)
    select_kernel(ctx, args.kernel or 4, args.min_blocks)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)
    cam = nb.city_camera(WIDTH // 2, HEIGHT // 2)
    prim = cam.primary_rays(SPP, seed=SEED + 10)
    d_p = torch.from_numpy(prim.view(np.float32).reshape(-1, 8)).cuda()
    h_p = torch.empty((prim.shape[0], 5), dtype=torch.int32, device="cuda")
    ctx.trace_closest_dev(d_p.data_ptr(), prim.shape[0], h_p.data_ptr())
    torch.cuda.synchronize()
    ph = h_p.cpu().numpy().view(nb.HIT_DTYPE).reshape(-1)
    bounce = nb.bounce_rays(prim, ph, sb.prims, seed=SEED + 11)
    d_b = torch.from_numpy(bounce.view(np.float32).reshape(-1, 8)).cuda()
    h_b = torch.empty((bounce.shape[0], 5), dtype=torch.int32, device="cuda")
    outs = []
    for _ in range(3):
        ctx.trace_closest_dev(d_p.data_ptr(), prim.shape[0], h_p.data_ptr())
        ctx.trace_closest_dev(d_b.data_ptr(), bounce.shape[0], h_b.data_ptr())
        torch.cuda.synchronize()
        outs.append((h_p.cpu().numpy(), h_b.cpu().numpy()))
    assert all(np.array_equal(o[0], outs[0][0]) and np.array_equal(o[1], outs[0][1]) for o in outs)
    assert ctx.status() == 0
    print(json.dumps({"profile_case": "city 960x540 x 4 spp primary, then bounce", "primary_rays": int(prim.shape[0]),
                      "bounce_rays": int(bounce.shape[0]), "kernel": nb.KERNEL_NAMES.get(args.kernel or 4)}))
    ctx.close()


def run_profile_compaction(args):
    """The device residency compaction of the 2.48M-triangle city under the bench's seeded 40 %
    object mask, three times; checks the three results agree."""
    import torch

    import nomad_b200 as nb

    sb = nb.SceneBVH(nb.synth_city(seed=SEED))
    rng = np.random.default_rng(SEED + 40)
    active = (rng.random(sb.object_count) < 0.4)[sb.prim_object].astype(np.uint8)
    comp = nb.native.Compactor(sb)
    act = torch.from_numpy(active).cuda()
    outs = []
    for _ in range(3):
        comp.run(act)
        torch.cuda.synchronize()
        outs.append(comp.result()["bvh_nodes"].view(np.uint32).copy())  # refs are int bits in float lanes
    assert all(np.array_equal(o, outs[0]) for o in outs)
    print(json.dumps({"profile_compaction": "city 2.48M triangles, 40 % of objects", "nodes": int(outs[0].size // 8)}))


def write_obj_scene(scene, folder):
    """Writes a HostScene's triangles as the reference's scene format: one OBJ file per object
    (unshared vertices relative to the object's centre, 1-based faces, a material library with
    a few materials), and a scene XML whose <Mesh> elements place each file at its centre.
    Returns the XML path and the bytes written."""
    geom = scene.prim_geom
    tri = scene.prim_type == 1
    lines_mtl = []
    for k in range(4):
        lines_mtl += [f"newmtl m{k}", f"Kd {0.2 + 0.2 * k:.2f} {0.5:.2f} {0.8 - 0.15 * k:.2f}",
                      f"Ns {10 * (k + 1)}", ""]
    total = 0
    with open(os.path.join(folder, "mats.mtl"), "w") as f:
        total += f.write("\n".join(lines_mtl))
    xml = ['<Scene width="1920" height="1080" maxRayDepth="3" residencyStrategy="alwaysresident">',
           '  <CameraPath><Keyframe frame="0" position="0,220,-620" lookAt="0,0,60"/></CameraPath>']
    for o in range(scene.object_count):
        a, n = int(scene.object_first[o]), int(scene.object_prims[o])
        g = geom[a:a + n][tri[a:a + n]]
        if g.shape[0] == 0:
            continue
        v = g[:, :9].reshape(-1, 3).astype(np.float64)
        c = v.mean(0)
        rel = v - c
        body = ["mtllib mats.mtl", f"o part{o}", f"usemtl m{o % 4}"]
        body += [f"v {x:.6f} {y:.6f} {z:.6f}" for x, y, z in rel]
        body += [f"f {3 * i + 1} {3 * i + 2} {3 * i + 3}" for i in range(g.shape[0])]
        with open(os.path.join(folder, f"obj{o}.obj"), "w") as f:
            total += f.write("\n".join(body) + "\n")
        xml.append(f'  <Mesh file="obj{o}.obj" position="{c[0]:.6f},{c[1]:.6f},{c[2]:.6f}" scale="1"/>')
    xml.append("</Scene>")
    path = os.path.join(folder, "scene.xml")
    with open(path, "w") as f:
        total += f.write("\n".join(xml) + "\n")
    return path, total


def ingest_leg(nb):
    """Scene ingest (nomad_scene_load_xml): the bench city's generator at 0.6M triangles written
    as the reference's XML scene format with one OBJ file per object, then read back on all host
    threads and on one; load
    time, triangles per second and OBJ text throughput. Parity with the reference's loader is
    checked by the tests and the oracle's scene recipe, not here."""
    import tempfile

    scene = nb.synth_city(seed=SEED, target_tris=600_000)
    with tempfile.TemporaryDirectory() as d:
        t0 = time.perf_counter()
        path, nbytes = write_obj_scene(scene, d)
        write_s = time.perf_counter() - t0
        out = {"workload": "city (1,024 objects, 0.6M triangles) as 1 XML + one OBJ per object "
                           "(unshared vertices) + 1 MTL",
               "bytes": nbytes, "write_s": write_s, "threads": len(os.sched_getaffinity(0))}
        for name, threads in (("all_threads", 0), ("one_thread", 1)):
            best = None
            for _ in range(2 if threads == 0 else 1):
                t0 = time.perf_counter()
                s = nb.load_scene_xml(path, threads=threads)
                dt = time.perf_counter() - t0
                best = dt if best is None else min(best, dt)
            out[name] = {"s": best, "mtris_per_s": s.prim_count / best / 1e6, "mb_per_s": nbytes / best / 1e6}
        out["triangles"], out["objects"], out["obj_files"] = s.prim_count, s.object_count, s.mesh_files
    return out


def select_kernel(ctx, kernel, min_blocks=0):
    """Fixes the traversal to a NOMAD_KERNEL_* variant, optionally with a min_blocks bound."""
    import nomad_b200 as nb

    ctx.set_kernel(kernel)
    if min_blocks:
        t = ctx.traversal()
        t["min_blocks"] = min_blocks
        ctx.set_traversal(**t)
    return nb.KERNEL_NAMES.get(kernel, str(kernel)) + (f"_mb{min_blocks}" if min_blocks else "")


def run_profile_frame(args):
    """Renders the city frame of the path-tracing leg twice (the second from the captured graph)
    with the chosen traversal variant (--kernel, default bvh4_persist)."""
    import torch

    import nomad_b200 as nb

    scene = nb.synth_city(seed=SEED)
    sb = nb.SceneBVH(scene)
    ctx = nb.Context(0)
    ctx.upload(sb)
    select_kernel(ctx, args.kernel or 4, args.min_blocks)
    v = nb.view_pinhole((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), width=WIDTH, height=HEIGHT, spp=SPP,
                        max_depth=3, seed=SEED)
    out = torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32, device="cuda")
    for f in range(2):
        v["frame"] = f
        ctx.render_dev(v, out.data_ptr())
    ctx.sync()
    assert ctx.status() == 0
    print(json.dumps({"profile_frame": "city 1920x1080 x 4 spp, 3 bounces", "stats": ctx.render_stats().tolist()}))
    ctx.close()


def run_profile_restir(args):
    """The ReSTIR leg's timing frame: city with 4,096 emissive triangles, 1920x1080 x 1 spp,
    direct lighting by ReSTIR (32 candidates, temporal + 3 spatial), three frames."""
    import torch

    import nomad_b200 as nb

    scene = nb.synth_city(seed=SEED, emissive_tris=4096, emissive_sigma=1.5)
    sb = nb.SceneBVH(scene)
    ctx = nb.Context(0)
    ctx.upload(sb)
    select_kernel(ctx, args.kernel or 4, args.min_blocks)
    ctx.set_restir(candidates=32, temporal=True, spatial=3, radius_px=30.0, m_cap=20.0)
    v = nb.view_pinhole((0.0, 220.0, -620.0), (0.0, 0.0, 60.0), width=WIDTH, height=HEIGHT, spp=1, max_depth=1,
                        seed=SEED, flags=nb.VIEW_RESTIR)
    out = torch.empty(WIDTH * HEIGHT * 3, dtype=torch.float32, device="cuda")
    for f in range(3):
        v["frame"] = f + 1
        ctx.render_dev(v, out.data_ptr())
    ctx.sync()
    assert ctx.status() == 0
    print(json.dumps({"profile_restir": "city + 4,096 emissive tris, 1920x1080 x 1 spp", "frames": 3}))
    ctx.close()


def ranks_max(x: float, world: int, device: str = "cuda") -> float:
    """The maximum of x over the ranks of the process group (x itself with one rank). A timing
    taken on every rank becomes the slowest rank's, as the whole job finishes with it."""
    if world <= 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job throughput in millions of units per second: every rank processes
    units_per_rank per step (weak scaling), the job lasts `seconds` (the slowest rank's)."""
    return world * units_per_rank * steps / seconds / 1e6


def run_reference(args):
    """The reference arm: the reference's own traversal (firstHitTLAS from PathTracing.h, compiled
    here from its sources into oracle/_ref) on all host threads, over the same workload, built
    without this repository's library (oracle/workload.py: the generator's source compiled on its
    own, the reference's own SceneBVH builder, numpy rays, the reference's own primary hits)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import reference as ref
    from oracle import workload as wl
    from nomad_b200.rays import city_camera  # numpy only: maps no library

    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (the reference compiled from its "
                          "sources) is not built"}), flush=True)
        return
    scene = wl.synth_city(seed=SEED)
    sb = wl.scene_bvh(scene)
    cores = len(os.sched_getaffinity(0))
    mix = wl.city_rays(sb, city_camera(WIDTH, HEIGHT), CONFIG["spp"], SEED + 10, SEED + 11, sample=400_000,
                       threads=cores)
    per_step = min(mix.shape[0], 300_000)
    for _ in range(args.warmup):
        ref.closest(sb, mix[:20_000], threads=cores)
    times = []
    for s in range(args.steps):
        part = mix[(s * per_step) % mix.shape[0]:][:per_step]
        t0 = time.perf_counter()
        ref.closest(sb, part, threads=cores)
        times.append((time.perf_counter() - t0, part.shape[0]))
    tot_t = sum(t for t, _ in times)
    tot_r = sum(n for _, n in times)
    v = tot_r / tot_t / 1e6
    line = {"impl": "reference", "metric": METRIC,
            "value": v, "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": dict(CONFIG, parallelism=f"replicas{world}"),
            "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": cores, "kind": "reference",
                             "sample": f"{per_step} rays per step from a 400,000-ray primary sample of the "
                                       f"workload and its bounces"},
            "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="nomad", choices=["nomad", "reference"])
    ap.add_argument("--kernel", type=int, default=0)
    ap.add_argument("--min-blocks", type=int, default=0,
                    help="with --kernel: resident blocks per SM the kernel is compiled for (0, 10, 12, 16)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the path-tracing, multi-view, ReSTIR and residency legs")
    ap.add_argument("--spp", type=int, default=SPP,
                    help="primary rays per pixel (smaller values give the profiling case)")
    ap.add_argument("--profile-compaction", action="store_true",
                    help="run only the device residency compaction of the city (for ncu)")
    ap.add_argument("--profile-case", action="store_true",
                    help="small case for ncu captures: the city, 960x540 x 4 spp primary rays and their "
                         "bounces as separate launches, three iterations of the chosen kernel (--kernel)")
    ap.add_argument("--profile-frame", action="store_true",
                    help="path-traced city frame (1920x1080 x 4 spp, 3 bounces) rendered twice, for launch lists")
    ap.add_argument("--profile-restir", action="store_true",
                    help="ReSTIR city (4,096 emissive triangles), 1920x1080 x 1 spp, three frames, for launch lists")
    args = ap.parse_args()
    CONFIG["spp"] = args.spp
    if args.impl == "reference":
        return run_reference(args)
    if args.profile_case:
        return run_profile_case(args)
    if args.profile_frame:
        return run_profile_frame(args)
    if args.profile_restir:
        return run_profile_restir(args)
    if args.profile_compaction:
        return run_profile_compaction(args)

    import torch
    import torch.distributed as dist
    import nomad_b200 as nb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    t_setup = time.perf_counter()
    scene, sb, primary = build_workload(nb, args.spp)
    ctx = nb.Context(local)
    ctx.upload(sb)
    if args.kernel:
        select_kernel(ctx, args.kernel, args.min_blocks)
    # A dedicated stream: the kernels and the timing events must share it (the legacy default
    # stream has handle 0, which the C ABI reads as "the context's own stream").
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    def dev_rays(r):
        return torch.from_numpy(r.view(np.float32).reshape(-1, 8)).cuda()

    d_prim = dev_rays(primary)
    d_ph = torch.empty((primary.shape[0], 5), dtype=torch.int32, device="cuda")
    ctx.trace_closest_dev(d_prim.data_ptr(), primary.shape[0], d_ph.data_ptr())
    torch.cuda.synchronize()
    ph = d_ph.cpu().numpy().view(nb.HIT_DTYPE).reshape(-1)
    bounce = nb.bounce_rays(primary, ph, sb.prims, seed=SEED + 11)
    d_b = dev_rays(bounce)
    d_bh = torch.empty((bounce.shape[0], 5), dtype=torch.int32, device="cuda")
    n_prim, n_b = primary.shape[0], bounce.shape[0]
    rays_per_step = n_prim + n_b
    log(f"setup {time.perf_counter() - t_setup:.1f}s: {sb.prim_count} prims, "
        f"{n_prim} primary + {n_b} bounce rays")

    # Algorithmic bytes per launch from the work counters (near-first binary traversal).
    d_w = torch.empty((max(n_prim, n_b), 4), dtype=torch.int32, device="cuda")

    def alg_bytes(d, n):
        ctx.trace_work_dev(d.data_ptr(), n, d_w.data_ptr())
        torch.cuda.synchronize()
        w = d_w[:n].to(torch.int64)
        return int((32 * w[:, 0] + 52 * w[:, 1] + 16 * w[:, 2] + 48 * w[:, 3]).sum().item())

    bytes_prim = alg_bytes(d_prim, n_prim)
    bytes_b = alg_bytes(d_b, n_b)
    del d_w

    # Autotune the traversal configuration on a sample of this frame's rays (1M primary + 1M
    # bounce): width x short stack x regroup threshold x staged top levels x block, each checked
    # bit for bit against the binary kernel.
    tune = None
    if args.kernel == 0:
        sample = torch.cat([d_prim[:1_000_000], d_b[:1_000_000]]).contiguous()
        torch.cuda.synchronize()
        sweep = ctx.autotune_sweep((sample.data_ptr(), sample.shape[0]), repeats=2, device=True)
        del sample
        rows = sorted((e for e in sweep["entries"] if e[2] >= 0), key=lambda e: e[2])
        tune = {"best": sweep["best_name"], "best_cfg": sweep["best"], "configs": len(sweep["entries"]),
                "mismatching_configs": sum(1 for e in sweep["entries"] if e[3]),
                "sample_rays": 2_000_000,
                "fastest_ms": [[e[0], round(e[2], 4)] for e in rows[:10]],
                "legacy_ms": {e[0]: round(e[2], 4) for e in sweep["entries"] if e[1]["persistent"] < 2},
                "slowest_ms": [[e[0], round(e[2], 4)] for e in rows[-3:]]}
        log(f"autotune: {tune}")

    def step():
        ctx.trace_closest_dev(d_prim.data_ptr(), n_prim, d_ph.data_ptr())
        ctx.trace_closest_dev(d_b.data_ptr(), n_b, d_bh.data_ptr())

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        time.sleep(0.5)
        torch.cuda.synchronize()
        t_begin = time.time()
        start.record(stream)
        for i in range(args.steps):
            ev[i][0].record(stream)
            ctx.trace_closest_dev(d_prim.data_ptr(), n_prim, d_ph.data_ptr())
            ev[i][1].record(stream)
            ctx.trace_closest_dev(d_b.data_ptr(), n_b, d_bh.data_ptr())
            ev[i][2].record(stream)
        end.record(stream)
        torch.cuda.synchronize()
        t_end = time.time()
        time.sleep(0.1)
    if world > 1:
        dist.barrier()
    total_ms = start.elapsed_time(end)
    t_prim = np.mean([e[0].elapsed_time(e[1]) for e in ev])
    t_b = np.mean([e[1].elapsed_time(e[2]) for e in ev])
    total_ms = ranks_max(total_ms, world)
    ms_step = total_ms / args.steps
    value = job_rate(world, rays_per_step, args.steps, total_ms / 1e3)

    # e2e through the C ABI with pinned host buffers (copies inside the timed region).
    h_rays = torch.from_numpy(np.concatenate([primary, bounce]).view(np.uint8)).pin_memory()
    h_hits = torch.empty((rays_per_step * 20,), dtype=torch.uint8).pin_memory()
    rays_np = h_rays.numpy().view(nb.RAY_DTYPE)
    hits_np = h_hits.numpy().view(nb.HIT_DTYPE)
    ctx.set_stream(0)

    def e2e_step():
        st = ctx.lib.nomad_trace_closest(ctx.h, rays_np.ctypes.data, rays_per_step,
                                         hits_np.ctypes.data, 0)
        if st != 0:
            raise nb.NomadError(st, ctx.lib.nomad_last_error(ctx.h).decode())

    for _ in range(2):
        e2e_step()
    if world > 1:
        dist.barrier()
    e_steps = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(e_steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_s = ranks_max(e2e_s, world)
    e2e_value = job_rate(world, rays_per_step, e_steps, e2e_s)
    ok = np.array_equal(hits_np.view(np.int32).reshape(-1, 5)[:n_prim],
                        d_ph.cpu().numpy()) if True else True

    peak, peak_kind = measured_peaks()
    achieved = (bytes_prim + bytes_b) / ((t_prim + t_b) / 1e3) / 1e9
    traffic = measured_traffic({"primary": n_prim, "bounce": n_b})
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak,
                # DRAM bytes of the step's two launches (primary + bounce), the launches `achieved`
                # covers: bytes per ray from a single-kernel ncu capture of the profile case
                # (profiles/), scaled by this step's rays
                "traffic": (traffic["primary"] + traffic["bounce"]) if traffic else None,
                "traffic_per_launch": traffic,
                "peak_source": peak_kind,
                "algorithmic_bytes_per_launch": {"primary": bytes_prim, "bounce": bytes_b},
                "kernel_ms": {"primary": t_prim, "bounce": t_b}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_leg(sb, np.concatenate([primary, bounce]))

    extras = {}
    if world > 1 and not args.no_extras:
        ctx.set_stream(0)
        try:
            extras["city_frame_split"] = split_frame_leg(nb, ctx, world)
        except Exception as exc:  # reported, never hiding the headline line
            extras["city_frame_split"] = {"error": repr(exc)}
    if rank == 0 and world == 1 and not args.no_extras:
        ctx.set_stream(0)
        for name, fn in (("city_frame", lambda: frame_leg(nb, ctx, sb)),
                         ("multiview", lambda: multiview_leg(nb, ctx)),
                         ("restir", lambda: restir_leg(nb, ctx)),
                         ("residency", lambda: residency_leg()),
                         ("compaction", lambda: compaction_leg(nb, sb, primary)),
                         ("ingest", lambda: ingest_leg(nb))):
            try:
                t0 = time.perf_counter()
                extras[name] = fn()
                log(f"{name}: {time.perf_counter() - t0:.1f}s {extras[name]}")
            except Exception as exc:  # an extra leg never hides the headline line
                extras[name] = {"error": repr(exc)}

    if rank == 0:
        line = {
            "metric": METRIC,
            "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(CONFIG, parallelism=f"replicas{world}"),
            "primary_mrays_s": n_prim / (t_prim / 1e3) / 1e6,
            "bounce_mrays_s": n_b / (t_b / 1e3) / 1e6,
            "rays_per_step": rays_per_step,
            "e2e": {"value": e2e_value, "unit": "Mrays/s",
                    "h2d_bytes_per_step": rays_per_step * 32, "d2h_bytes_per_step": rays_per_step * 20,
                    "matches_device_result": bool(ok)},
            "gpu_launches": 2 * args.steps,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": clk.summary(t_begin, t_end),
            "kernel_variant": tune["best"] if tune else nb.KERNEL_NAMES.get(args.kernel, str(args.kernel)) + (
                f"_mb{args.min_blocks}" if args.min_blocks else ""),
            "autotune": tune,
        }
        line.update(extras)
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
