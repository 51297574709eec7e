"""GPU tests of the device residency step and the learned BF16 MLP scorer.

* MLP inference against a float64 restatement with the device's bf16 roundings
  (tolerance 1e-3 relative: only the fp32 accumulation order differs);
* training lowers the loss and is bit-reproducible for a seed; the weight blob round-trips;
* the residency step's keys, selection under a byte budget and TLAS patching against the
  oracle restatement; traversal and rendering after eviction against the oracle.
"""
import numpy as np
import pytest

from tests import raysets

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(nb):
    c = nb.Context(0)
    yield c
    c.close()


def _features(n, seed):
    rng = np.random.default_rng(seed)
    f = rng.normal(size=(n, 24)).astype(np.float32) * 2.0 + 1.0
    return f


def test_mlp_forward_matches_restatement(nb, ctx, small_city):
    from oracle import residency as ores

    ctx.upload(small_city[1])
    ctx.mlp_init(123)
    x = _features(1000, 1)
    got = ctx.mlp_infer(x)
    want = ores.mlp_forward(ctx.mlp_get(), x)
    err = np.abs(got - want) / (1.0 + np.abs(want))
    assert err.max() < 1e-3, err.max()
    # tensor-memory waits of the tcgen05 inference kernel all completed
    assert ctx.status() == 0


def test_mlp_training(nb, ctx, small_city):
    from oracle import residency as ores

    ctx.upload(small_city[1])
    rng = np.random.default_rng(2)
    x = _features(16384, 3)
    t = np.log1p(np.abs(x[:, 0] * 2 + x[:, 5] - 0.5 * x[:, 11] ** 2)).astype(np.float32)
    ctx.mlp_init(7)
    loss = ctx.mlp_train(x, t, steps=300, batch=1024, lr=2e-3, seed=11)
    assert np.isfinite(loss).all()
    assert loss[-20:].mean() < 0.25 * loss[:5].mean(), (loss[:5], loss[-20:])
    blob = ctx.mlp_get()
    # reproducible: same seed, same weights
    ctx.mlp_init(7)
    ctx.mlp_train(x, t, steps=300, batch=1024, lr=2e-3, seed=11)
    assert np.array_equal(ctx.mlp_get(), blob)
    # checkpoint round trip
    pred = ctx.mlp_infer(x[:500])
    ctx.mlp_init(99)
    ctx.mlp_set(blob)
    assert np.array_equal(ctx.mlp_infer(x[:500]), pred)
    err = np.abs(pred - ores.mlp_forward(blob, x[:500])) / (1.0 + np.abs(pred))
    assert err.max() < 1e-3


def _residency_frame(nb, ctx, view):
    ctx.reset_object_hits()
    ctx.render(view, count_hits=True)
    return ctx.object_hits().astype(np.int64)


@pytest.mark.parametrize("bonus", [0.0, 0.5])
@pytest.mark.parametrize("sync_toggles", [True, False])
@pytest.mark.parametrize("policy", [0, 1, 2])
def test_residency_step_against_oracle(nb, orc, ctx, small_city, policy, sync_toggles, bonus):
    """The device step against the restatement over a moving camera; bonus > 0 is the selection's
    hysteresis (resident keys raised by bonus * |key|)."""
    from oracle import residency as ores

    if policy == 0 and bonus:
        pytest.skip("AlwaysResident has no keys")

    scene, sb = small_city
    ctx.upload(sb)
    if policy == nb.POLICY_LEARNED:
        ctx.mlp_init(5)
    nbytes = ctx.object_bytes()
    budget = int(0.4 * nbytes.sum())
    prm = nb.ResidencyParams.make(policy, budget_bytes=budget, camera_motion=0.5, memory_pressure=0.25,
                                  min_active=2, resident_key_bonus=bonus)
    score = np.zeros(sb.object_count, np.float64)
    flags = np.ones(sb.object_count, np.uint8)
    for frame, pos in enumerate([(0, 60, -180), (20, 50, -150), (40, 45, -120)]):
        view = nb.view_pinhole(pos, (0, 0, 0), width=96, height=54, spp=2, max_depth=2, seed=frame)
        hits = _residency_frame(nb, ctx, view)
        toggles = ctx.residency_step(prm, view, toggles=sync_toggles)
        feats, keys = ctx.residency_last()
        score = (score.astype(np.float32) * np.float32(0.85) + hits.astype(np.float32)).astype(np.float32)
        visible = feats[:, 2] > 0.5
        if policy == nb.POLICY_RAYHIT_BUDGET:
            want_keys = ores.rayhit_keys(score, hits, visible, 0.25)
            assert np.array_equal(keys, want_keys)
        if policy == nb.POLICY_LEARNED:
            want_keys = ctx.mlp_infer(feats)
            assert np.array_equal(keys, want_keys)
        reserve = ores.reserve_count(sb.object_count, 0.02, 0.06, 0.5)
        want, want_t = ores.select(keys, visible, nbytes, budget, reserve, 2, flags,
                                   always=(policy == nb.POLICY_ALWAYS), resident_bonus=bonus)
        got = ctx.residency_flags()
        assert np.array_equal(got, want), (frame, np.nonzero(got != want)[0][:10])
        assert toggles == (want_t if sync_toggles else None)
        flags = got
        if policy != nb.POLICY_ALWAYS:
            assert int(nbytes[flags.astype(bool)].sum()) <= budget + int(np.sort(nbytes)[-2:].sum())
    inst = ctx.instances()
    root = sb.instances["blas_root_index"].copy()
    root[flags == 0] = -1
    assert np.array_equal(inst["blas_root_index"], root)
    # traversal and shading see exactly the resident set
    rays = np.concatenate([raysets.aimed_rays(sb, 8000, 1), raysets.random_rays(sb, 4000, 2)])
    ref = orc.OracleScene(sb, blas_root=root)
    got = ctx.trace_closest(rays)
    assert np.array_equal(np.ascontiguousarray(got).view(np.int32), np.ascontiguousarray(ref.closest(rays)).view(np.int32))
    v = nb.view_pinhole((0, 60, -180), (0, 0, 0), width=48, height=27, spp=2, max_depth=3, seed=9)
    img = ctx.render(v)[0].reshape(-1, 3)
    want_img, _, _ = orc.render(ref, sb.materials, v)
    assert (img == want_img).all(1).mean() > 0.99


@pytest.mark.parametrize("policy", [1, 2])
def test_residency_step_many_objects(nb, orc, ctx, policy):
    """2,048 objects (the learned-residency object count): the selection kernel's block-parallel
    budget walks span several sorted positions per thread; flags must equal the restatement."""
    from oracle import residency as ores

    scene = nb.synth_city(seed=31, grid=64, grid_z=32, size_m=2000.0, target_tris=150_000, median_tris=60,
                          max_tris=2_000, emissive_quads=16)
    sb = nb.SceneBVH(scene)
    assert sb.object_count >= 2048
    ctx.upload(sb)
    if policy == nb.POLICY_LEARNED:
        ctx.mlp_init(3)
    nbytes = ctx.object_bytes()
    for frac in (0.4, 0.1):
        budget = int(frac * nbytes.sum())
        prm = nb.ResidencyParams.make(policy, budget_bytes=budget, camera_motion=0.7, memory_pressure=0.5,
                                      min_active=5)
        flags = ctx.residency_flags()
        for frame, pos in enumerate([(0, 80, -900), (100, 60, -700)]):
            view = nb.view_pinhole(pos, (0, 0, 0), width=96, height=54, spp=2, max_depth=2, seed=frame)
            ctx.reset_object_hits()
            ctx.render(view, count_hits=True)
            toggles = ctx.residency_step(prm, view)
            feats, keys = ctx.residency_last()
            visible = feats[:, 2] > 0.5
            reserve = ores.reserve_count(sb.object_count, 0.02, 0.06, 0.7)
            want, want_t = ores.select(keys, visible, nbytes, budget, reserve, 5, flags)
            got = ctx.residency_flags()
            assert np.array_equal(got, want), (frac, frame, np.nonzero(got != want)[0][:10])
            assert toggles == want_t
            flags = got
    assert ctx.status() == 0


@pytest.mark.parametrize("max_toggles", [16, 0])
def test_rayhit_per_primitive_policy(nb, ctx, small_city, max_toggles):
    """The reference's per-primitive ray-hit budget (NOMAD_POLICY_RAYHIT_PRIM) against the numpy
    restatement frame by frame: decayed scores bit for bit, the same primitives toggled (budget,
    cooldowns, rebuild cooldown), the frustum test equal to a float64 restatement except within
    1e-4 rad of its boundary, and traversal after the toggles equal to the same activity set by hand."""
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    prm = nb.ResidencyParams.make(nb.POLICY_RAYHIT_PRIM, max_toggles=max_toggles, camera_motion=0.3,
                                  memory_pressure=0.2, min_active=16, target_fraction=0.54)
    view0 = nb.view_pinhole((0, 60, -180), (0, 0, 0), width=96, height=54, spp=2, max_depth=2, seed=1)
    ctx.residency_step(prm, view0)  # enables per-primitive counting (no hits yet)
    _, sc0, cd0, _, act0 = ctx.residency_prim_state()
    orc = ores.RayHitPrimOracle(sb.prim_count, act0)
    orc.score, orc.cooldown = sc0.copy(), cd0.copy()
    orc.rebuild = 0 if (act0 == 1).all() else 4
    spheres = ores.prim_spheres(sb.prims)
    for frame in range(8):
        ang = 0.25 * frame
        view = nb.view_pinhole((180 * np.sin(ang), 60, -180 * np.cos(ang)), (0, 0, 0), width=96, height=54,
                               spp=2, max_depth=2, seed=frame + 2)
        ctx.render(view, count_hits=True)
        hits, _, _, _, _ = ctx.residency_prim_state()
        assert hits.sum() > 0
        toggled = ctx.residency_step(prm, view)
        _, sc, cd, vis, act = ctx.residency_prim_state()
        want_toggles = orc.step(hits, vis, decay=0.85, motion=0.3, pressure=0.2, target_fraction=0.54,
                                max_toggles=max_toggles, min_active=16)
        assert np.array_equal(sc.view(np.uint32), orc.score.view(np.uint32)), frame
        assert toggled == want_toggles, (frame, toggled, want_toggles)
        assert np.array_equal(act, orc.active), frame
        assert np.array_equal(cd, orc.cooldown), frame
        if orc.ran:
            v64, margin = ores.in_view_f64(spheres, view)
            assert ((vis.astype(bool) == v64) | (margin < 1e-4)).all(), frame
    # traversal with the policy's activity equals the same activity set primitive by primitive
    rays = raysets.aimed_rays(sb, 4000, 3)
    got = ctx.trace_closest(rays)
    c2 = nb.Context(0)
    try:
        c2.upload(sb)
        for p in np.nonzero(act == 0)[0]:
            c2.set_primitive_active(int(p), False)
        c2.flush()
        want = c2.trace_closest(rays)
    finally:
        c2.close()
    assert np.array_equal(np.ascontiguousarray(got).view(np.int32), np.ascontiguousarray(want).view(np.int32))


def test_distance_lod_policy(nb, ctx, small_city):
    """The reference's DistanceLOD heuristic (NOMAD_POLICY_DISTANCE_LOD) against the numpy
    restatement over a camera fly-through: distances and frustum tests equal to a float64
    restatement (up to float32 rounding and 1e-4 rad at the frustum boundary), the same objects
    toggled (nearest first, hysteresis, cooldowns, toggle budget), traversal equal to the same
    residency set by hand."""
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    prm = nb.ResidencyParams.make(nb.POLICY_DISTANCE_LOD, max_toggles=6, camera_motion=0.2, memory_pressure=0.1,
                                  lod_enter_distance=90.0, lod_exit_distance=120.0)
    orc = ores.DistanceLodOracle(sb.object_count, sb.instances["primitive_count"])
    spheres = ores.object_spheres(sb)
    total = 0
    for frame in range(10):
        x = -120.0 + 24.0 * frame
        view = nb.view_pinhole((x, 30, -60), (x + 10, 0, 60), width=96, height=54, spp=1, max_depth=1, seed=frame)
        toggled = ctx.residency_step(prm, view)
        dist, flags, cd = ctx.residency_object_state()
        d64, en, ex, be, margin = ores.lod_tests_f64(spheres.astype(np.float64), view)
        ok = np.abs(dist.astype(np.float64) - d64) <= 1e-3 * np.maximum(1.0, d64)
        assert (ok | (dist == np.finfo(np.float32).max)).all(), frame
        f64 = (en.astype(np.uint8) | (ex.astype(np.uint8) << 1) | (be.astype(np.uint8) << 2))
        assert ((flags == f64) | (margin < 1e-4)).all(), frame
        want = orc.step(dist, flags, motion=0.2, pressure=0.1, max_toggles=6, enter=90.0, exit_=120.0)
        assert toggled == want, (frame, toggled, want)
        assert np.array_equal(cd, orc.cooldown), frame
        assert np.array_equal(ctx.residency_flags().astype(bool), orc.active_count > 0), frame
        total += toggled
    assert total > 0
    rays = raysets.aimed_rays(sb, 4000, 5)
    got = ctx.trace_closest(rays)
    flags_obj = ctx.residency_flags()
    c2 = nb.Context(0)
    try:
        c2.upload(sb)
        for o in np.nonzero(flags_obj == 0)[0]:
            c2.set_object_active(int(o), False)
        c2.flush()
        want_h = c2.trace_closest(rays)
    finally:
        c2.close()
    assert np.array_equal(np.ascontiguousarray(got).view(np.int32), np.ascontiguousarray(want_h).view(np.int32))


def test_screen_space_policy(nb, ctx, small_city):
    """The reference's ScreenSpaceFootprint heuristic (NOMAD_POLICY_SCREEN_SPACE) against the numpy
    restatement over a camera orbit: coverage equal to a float64 restatement (relative 1e-3, or a
    decision within 1e-4 of its boundary), the same objects toggled under the primitive budget and
    cooldowns."""
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    prm = nb.ResidencyParams.make(nb.POLICY_SCREEN_SPACE, max_toggles=3000, camera_motion=0.2, memory_pressure=0.1,
                                  target_fraction=0.6, min_active=16, min_pixel_coverage=32.0)
    orc = ores.ScreenSpaceOracle(sb.instances["primitive_count"])
    spheres = ores.object_spheres(sb)
    total = 0
    for frame in range(10):
        ang = 0.3 * frame
        view = nb.view_pinhole((160 * np.sin(ang), 70, -160 * np.cos(ang)), (0, 0, 0), width=128, height=72, spp=1,
                               max_depth=1, seed=frame)
        toggled = ctx.residency_step(prm, view)
        cov, _, cd = ctx.residency_object_state()
        c64, margin = ores.coverage_f64(spheres, view)
        ok = np.abs(cov.astype(np.float64) - c64) <= 1e-3 * np.maximum(1.0, c64)
        assert (ok | (margin < 1e-4)).all(), frame
        want = orc.step(cov, 128, 72, motion=0.2, pressure=0.1, target_fraction=0.6, min_pixel=32.0, min_active=16,
                        max_toggles=3000)
        assert toggled == want, (frame, toggled, want)
        assert np.array_equal(ctx.residency_flags().astype(bool), orc.active), frame
        assert np.array_equal(cd, orc.cooldown), frame
        total += toggled
    assert total > 0


def test_mlp_gradient_and_adamw_match_restatement(nb, ctx, small_city):
    """The training kernels against a float64 restatement with the device's BF16 roundings: the
    gradient of every parameter group (W1, b1, W2, b2, w3, b3) from nomad_mlp_gradient, and the
    parameters after one and after two AdamW steps of nomad_mlp_train on the whole batch."""
    from oracle import residency as ores

    ctx.upload(small_city[1])
    B = 512
    x = _features(B, 9)
    t = np.log1p(np.abs(x[:, 0] * 2 + x[:, 5] - 0.5 * x[:, 11] ** 2)).astype(np.float32)
    ctx.mlp_init(3)
    ctx.mlp_train(x, t, steps=0, batch=B)  # stores the feature statistics only
    blob0 = ctx.mlp_get()
    g, loss = ctx.mlp_gradient(x, t)
    r, rloss = ores.mlp_gradient(blob0, x, t)
    assert abs(loss - rloss) <= 1e-4 * rloss
    o = ores._blob_parts(blob0)
    groups = [("w1", "b1"), ("b1", "w2"), ("w2", "b2"), ("b2", "w3"), ("w3", "b3")]
    for a, b in groups + [("b3", None)]:
        lo, hi = o[a], (o[b] if b else o[a] + 1)
        ga, ra = g[lo:hi].astype(np.float64), r[lo:hi]
        scale = np.abs(ra).max()
        assert scale > 0 and np.abs(ga - ra).max() <= 2e-3 * scale, (a, np.abs(ga - ra).max(), scale)
    assert (g[o["mean"]:] == 0).all() and (g[:o["b1"]].reshape(128, 32)[:, 24:] == 0).all()
    # AdamW: one step, then two steps from the same start (each call starts fresh moments); the
    # second step's gradient is restated at the device's parameters after the first
    lr, wd = 2e-3, 1e-2
    ctx.mlp_train(x, t, steps=1, batch=B, lr=lr, weight_decay=wd, seed=5)
    blob1 = ctx.mlp_get()
    z = np.zeros(blob0.size, np.float32)
    want1, m1, v1 = ores.adamw_step(blob0, r, z, z, 1, lr, wd)
    sig = np.abs(r[:o["mean"]]) > 1e-3 * np.abs(r[:o["mean"]]).max()  # sign(g) decides step 1
    assert np.abs(blob1 - want1)[:o["mean"]][sig].max() <= 1e-6
    assert np.array_equal(blob1[o["mean"]:], blob0[o["mean"]:])
    ctx.mlp_set(blob0)
    ctx.mlp_train(x, t, steps=2, batch=B, lr=lr, weight_decay=wd, seed=5)
    blob2 = ctx.mlp_get()
    r1, _ = ores.mlp_gradient(blob1, x, t)
    want2, _, _ = ores.adamw_step(blob1, r1, m1, v1, 2, lr, wd)
    big = np.abs(r1[:o["mean"]]) > 1e-2 * np.abs(r1[:o["mean"]]).max()
    assert np.abs(blob2 - want2)[:o["mean"]][big].max() <= 1e-5
    assert np.median(np.abs(blob2 - want2)[:o["mean"]]) <= 1e-6
