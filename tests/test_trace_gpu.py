"""GPU parity: the CUDA traversal against the scalar oracle, through the C ABI.

Bar: (instance, primitive) bit-exact, and t/u/v bit-exact too (the kernels use the oracle's
operation order with no FMA, so the 4-ulp allowance is not needed); any-hit booleans
bit-exact; per-object hit counters equal to the oracle's per-object sums.
"""
import numpy as np
import pytest

from tests import raysets

pytestmark = pytest.mark.gpu


def _bits(h):
    return np.ascontiguousarray(h).view(np.int32).reshape(-1, 5)


def _assert_hits_equal(got, want):
    g, w = _bits(got), _bits(want)
    bad = np.nonzero((g != w).any(1))[0]
    assert bad.size == 0, f"{bad.size} of {len(g)} rays differ; first {bad[:5]}: got {got[bad[:3]]} want {want[bad[:3]]}"


def _rays(sb, seed, n=20000):
    return np.concatenate([raysets.aimed_rays(sb, n, seed), raysets.random_rays(sb, n, seed + 1),
                           raysets.edge_case_rays(sb, seed + 2)])


@pytest.fixture(scope="module")
def ctx(nb):
    c = nb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("kernel", [1, 2, 3, 4, 5, 6])
@pytest.mark.parametrize("which", ["ico", "city"])
def test_closest_parity(nb, orc, ctx, ico_scene, small_city, which, kernel):
    scene, sb = ico_scene if which == "ico" else small_city
    ctx.upload(sb)
    ctx.set_kernel(kernel)
    cam = nb.icosphere_camera(160, 90) if which == "ico" else nb.Camera((0, 60, -180), (0, 0, 0), width=160, height=90)
    prim = cam.primary_rays(2, seed=3)
    rays = np.concatenate([prim, _rays(sb, 40)])
    ref = orc.OracleScene(sb)
    want = ref.closest(rays)
    got = ctx.trace_closest(rays)
    _assert_hits_equal(got, want)
    bounce = nb.bounce_rays(prim, want[: prim.shape[0]], sb.prims, seed=4)
    _assert_hits_equal(ctx.trace_closest(bounce), ref.closest(bounce))
    assert ctx.status() == 0
    ctx.set_kernel(1)


@pytest.mark.parametrize("kernel", [1, 3, 5])
@pytest.mark.parametrize("which", ["ico", "city"])
def test_any_parity(orc, ctx, ico_scene, small_city, which, kernel):
    scene, sb = ico_scene if which == "ico" else small_city
    ctx.upload(sb)
    ctx.set_kernel(kernel)
    rays = _rays(sb, 50)
    # finite tmax: half of each ray's closest distance, so some rays become unoccluded
    ref = orc.OracleScene(sb)
    h = ref.closest(rays)
    short = rays.copy()
    hit = h["prim"] >= 0
    short["tmax"][hit] = h["t"][hit] * np.float32(0.5)
    for rs in (rays, short):
        got = ctx.trace_any(rs)
        want = ref.any(rs)
        assert np.array_equal(got, want), f"{(got != want).sum()} any-hit mismatches"
    ctx.set_kernel(1)


def test_work_counters(orc, ctx, small_city):
    scene, sb = small_city
    ctx.upload(sb)
    rays = _rays(sb, 60, n=5000)
    w_ref, h_ref = orc.OracleScene(sb).work(rays)
    w = ctx.trace_work(rays)
    assert np.array_equal(w, w_ref)


def test_object_hit_counters(orc, ctx, small_city):
    scene, sb = small_city
    ctx.upload(sb)
    rays = _rays(sb, 70)
    ctx.reset_object_hits()
    h = ctx.trace_closest(rays, count_hits=True)
    h2 = ctx.trace_closest(rays[::3], count_hits=True)
    want = (np.bincount(h["inst"][h["prim"] >= 0], minlength=sb.object_count)
            + np.bincount(h2["inst"][h2["prim"] >= 0], minlength=sb.object_count))
    assert np.array_equal(ctx.object_hits(), want.astype(np.uint32))
    ctx.reset_object_hits()
    assert ctx.object_hits().sum() == 0


@pytest.mark.parametrize("kernel", [1, 4, 5])
def test_residency_toggles(orc, ctx, small_city, kernel):
    scene, sb = small_city
    ctx.upload(sb)
    ctx.set_kernel(kernel)
    rays = _rays(sb, 80)
    rng = np.random.default_rng(9)
    off_objs = np.nonzero(rng.random(sb.object_count) < 0.3)[0]
    off_prims = np.nonzero(rng.random(sb.prim_count) < 0.1)[0]
    toggled = sum(ctx.set_object_active(int(o), False) for o in off_objs)
    assert toggled == int(sb.instances["primitive_count"][off_objs].sum())
    for p in off_prims:
        ctx.set_primitive_active(int(p), False)
    ctx.flush()
    active = np.ones(sb.prim_count, np.uint8)
    active[off_prims] = 0
    for o in off_objs:
        b = sb.instances["primitive_base"][o]
        active[b:b + sb.instances["primitive_count"][o]] = 0
    root = sb.instances["blas_root_index"].copy()
    counts = np.add.reduceat(active.astype(np.int64), sb.instances["primitive_base"].astype(np.int64))
    root[counts == 0] = -1
    inst = ctx.instances()
    assert np.array_equal(inst["blas_root_index"], root)
    ref = orc.OracleScene(sb, active=active, blas_root=root)
    _assert_hits_equal(ctx.trace_closest(rays), ref.closest(rays))
    assert np.array_equal(ctx.trace_any(rays), ref.any(rays))
    # everything back on
    for o in range(sb.object_count):
        ctx.set_object_active(o, True)
    ctx.flush()
    _assert_hits_equal(ctx.trace_closest(rays), orc.OracleScene(sb).closest(rays))
    ctx.set_kernel(1)


def test_autotune(nb, orc, ctx, small_city):
    scene, sb = small_city
    ctx.upload(sb)
    rays = _rays(sb, 110)
    res = ctx.autotune(rays, repeats=2)
    assert all(v == 0 for v in res["mismatches"].values()), res
    assert res["ms"][res["best"]] > 0
    _assert_hits_equal(ctx.trace_closest(rays), orc.OracleScene(sb).closest(rays))
    ctx.set_kernel(1)


def test_device_pointer_path(nb, orc, ctx, small_city):
    import torch

    scene, sb = small_city
    ctx.upload(sb)
    rays = _rays(sb, 90)
    d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
    d_hits = torch.empty((rays.shape[0], 5), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    ctx.trace_closest_dev(d_rays.data_ptr(), rays.shape[0], d_hits.data_ptr())
    torch.cuda.synchronize()
    ctx.set_stream(0)
    got = d_hits.cpu().numpy().view(nb.HIT_DTYPE).reshape(-1)
    _assert_hits_equal(got, orc.OracleScene(sb).closest(rays))


def test_full_city_sample(nb, orc, ctx):
    """The 2.5M-triangle city at 1080p: a seeded 1/40 sample of the primary rays and their
    bounces against the oracle, and counters over all primary rays against the hits."""
    scene = nb.synth_city(seed=2)
    sb = nb.SceneBVH(scene)
    ctx.upload(sb)
    cam = nb.city_camera(1920, 1080)
    rays = cam.primary_rays(1, seed=5)
    ctx.reset_object_hits()
    hits = ctx.trace_closest(rays, count_hits=True)
    want = np.bincount(hits["inst"][hits["prim"] >= 0], minlength=sb.object_count)
    assert np.array_equal(ctx.object_hits(), want.astype(np.uint32))
    idx = np.random.default_rng(1).choice(rays.shape[0], rays.shape[0] // 40, replace=False)
    ref = orc.OracleScene(sb)
    _assert_hits_equal(hits[idx], ref.closest(rays[idx]))
    b = nb.bounce_rays(rays[idx], hits[idx], sb.prims, seed=6)
    _assert_hits_equal(ctx.trace_closest(b), ref.closest(b))
    assert ctx.status() == 0


# Short-stack persistent kernels: lane refill threshold, shared-memory short stack with local
# spill, staged top levels. Every configuration must return the oracle's hits bit for bit.
_RG_CONFIGS = [
    dict(width=2, short_stack=8, regroup=1, staged=False, block=128, post=0),
    dict(width=2, short_stack=0, regroup=24, staged=True, block=256, post=1),
    dict(width=2, short_stack=16, regroup=32, staged=True, block=256, post=0),
    dict(width=4, short_stack=8, regroup=16, staged=True, block=128, post=1),
    dict(width=4, short_stack=32, regroup=24, staged=False, block=256, post=0),
    dict(width=4, short_stack=0, regroup=32, staged=False, block=128, post=1),
    dict(width=8, short_stack=8, regroup=32, staged=True, block=256, post=0),
    dict(width=8, short_stack=16, regroup=1, staged=False, block=64, post=1),
]


def _set_rg(ctx, c):
    tl = ctx.tlas_nodes()[{2: 0, 4: 1, 8: 2}[c["width"]]]
    cap = (32 * 1024) // {2: 64, 4: 128, 8: 256}[c["width"]]
    ctx.set_traversal(width=c["width"], persistent=2, short_stack=c["short_stack"], regroup=c["regroup"],
                      staged_nodes=min(tl, cap) if c["staged"] else 0, block=c["block"],
                      postpone_leaves=c["post"])


@pytest.mark.parametrize("cfg", _RG_CONFIGS, ids=lambda c: "w{width}_ss{short_stack}_rg{regroup}_st{staged:d}_b{block}_p{post}".format(**c))
@pytest.mark.parametrize("which", ["ico", "city"])
def test_regroup_parity(nb, orc, ctx, ico_scene, small_city, which, cfg):
    scene, sb = ico_scene if which == "ico" else small_city
    ctx.upload(sb)
    _set_rg(ctx, cfg)
    cam = nb.icosphere_camera(160, 90) if which == "ico" else nb.Camera((0, 60, -180), (0, 0, 0), width=160, height=90)
    prim = cam.primary_rays(2, seed=13)
    rays = np.concatenate([prim, _rays(sb, 140)])
    ref = orc.OracleScene(sb)
    want = ref.closest(rays)
    ctx.reset_object_hits()
    got = ctx.trace_closest(rays, count_hits=True)
    _assert_hits_equal(got, want)
    counts = np.bincount(want["inst"][want["prim"] >= 0], minlength=sb.object_count).astype(np.uint32)
    assert np.array_equal(ctx.object_hits(), counts)
    bounce = nb.bounce_rays(prim, want[: prim.shape[0]], sb.prims, seed=14)
    _assert_hits_equal(ctx.trace_closest(bounce), ref.closest(bounce))
    short = rays.copy()
    hit = want["prim"] >= 0
    short["tmax"][hit] = want["t"][hit] * np.float32(0.5)
    for rs in (rays, short):
        assert np.array_equal(ctx.trace_any(rs), ref.any(rs))
    assert ctx.status() == 0
    ctx.set_kernel(1)


def test_regroup_residency(nb, orc, ctx, small_city):
    scene, sb = small_city
    ctx.upload(sb)
    _set_rg(ctx, dict(width=4, short_stack=16, regroup=24, staged=True, block=128, post=1))
    rays = _rays(sb, 150)
    rng = np.random.default_rng(19)
    off_objs = np.nonzero(rng.random(sb.object_count) < 0.4)[0]
    for o in off_objs:
        ctx.set_object_active(int(o), False)
    ctx.flush()
    root = sb.instances["blas_root_index"].copy()
    root[off_objs] = -1
    ref = orc.OracleScene(sb, blas_root=root)
    _assert_hits_equal(ctx.trace_closest(rays), ref.closest(rays))
    assert np.array_equal(ctx.trace_any(rays), ref.any(rays))
    for o in off_objs:
        ctx.set_object_active(int(o), True)
    ctx.flush()
    _assert_hits_equal(ctx.trace_closest(rays), orc.OracleScene(sb).closest(rays))
    ctx.set_kernel(1)


def test_autotune_sweep(nb, orc, ctx, small_city):
    scene, sb = small_city
    ctx.upload(sb)
    rays = _rays(sb, 160)
    res = ctx.autotune_sweep(rays, repeats=1)
    names = [e[0] for e in res["entries"]]
    assert len(names) > 300 and len(set(names)) == len(names)
    assert {"bvh2_packet", "bvh4_packet", "bvh8_packet"} <= set(names)
    assert all(e[3] == 0 for e in res["entries"] if e[2] >= 0), [e for e in res["entries"] if e[3]]
    assert {e[1]["width"] for e in res["entries"]} == {2, 4, 8}
    assert {e[1]["short_stack"] for e in res["entries"]} == {0, 8, 16, 32}
    assert ctx.traversal() == res["best"]
    _assert_hits_equal(ctx.trace_closest(rays), orc.OracleScene(sb).closest(rays))
    ctx.set_kernel(1)


@pytest.mark.parametrize("width", [2, 4, 8])
@pytest.mark.parametrize("which", ["ico", "city"])
def test_packet_parity(nb, orc, ctx, ico_scene, small_city, which, width):
    """Hybrid packet kernel: coherent warps (primary rays) walk as packets, the rest per ray."""
    scene, sb = ico_scene if which == "ico" else small_city
    ctx.upload(sb)
    ctx.set_traversal(width=width, persistent=3)
    cam = nb.icosphere_camera(160, 90) if which == "ico" else nb.Camera((0, 60, -180), (0, 0, 0), width=160, height=90)
    prim = cam.primary_rays(4, seed=23)
    rays = np.concatenate([prim, _rays(sb, 170)])
    ref = orc.OracleScene(sb)
    want = ref.closest(rays)
    ctx.reset_object_hits()
    _assert_hits_equal(ctx.trace_closest(rays, count_hits=True), want)
    counts = np.bincount(want["inst"][want["prim"] >= 0], minlength=sb.object_count).astype(np.uint32)
    assert np.array_equal(ctx.object_hits(), counts)
    short = rays.copy()
    hit = want["prim"] >= 0
    short["tmax"][hit] = want["t"][hit] * np.float32(0.5)
    for rs in (rays, short):
        assert np.array_equal(ctx.trace_any(rs), ref.any(rs))
    assert ctx.status() == 0
    ctx.set_kernel(1)


def test_full_city_variants(nb, orc, ctx):
    """The 2.5M-triangle city: a contiguous block of 1080p primary rays (coherent warps, so the
    packet walks run) and their bounces through every kernel family against the oracle."""
    scene = nb.synth_city(seed=2)
    sb = nb.SceneBVH(scene)
    ctx.upload(sb)
    rays = nb.city_camera(1920, 1080).primary_rays(1, seed=5)[700_000:760_000]
    ref = orc.OracleScene(sb)
    want = ref.closest(rays)
    b = nb.bounce_rays(rays, want, sb.prims, seed=8)
    want_b = ref.closest(b)
    sh = nb.shadow_rays(rays, want, sb.prims, sb.materials, seed=9)
    want_s = ref.any(sh)
    assert 0.05 < want_s.mean() < 0.999
    configs = [dict(width=w, persistent=3) for w in (2, 4, 8)]
    configs += [dict(width=w, persistent=2, short_stack=s, regroup=24, postpone_leaves=1) for w, s in ((2, 8), (4, 0), (8, 16))]
    configs += [dict(width=w, persistent=1, min_blocks=10) for w in (2, 4, 8)]
    for c in configs:
        ctx.set_traversal(**c)
        _assert_hits_equal(ctx.trace_closest(rays), want)
        _assert_hits_equal(ctx.trace_closest(b), want_b)
        assert np.array_equal(ctx.trace_any(sh), want_s), c
        assert ctx.status() == 0, c
    ctx.set_kernel(1)
