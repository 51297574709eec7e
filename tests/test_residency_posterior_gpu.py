"""The per-object hit-probability posterior and the policies built on it, on B200 against the
oracle's restatements:

* "rays tested" per object (closest-hit segments that enter the object's TLAS leaf box before
  their hit), counted by the device TLAS walk, against the oracle's test of every leaf box;
* processRayHitCounters' Beta posterior (alpha, beta, probability, variance, mass, exploration),
  updated by the device step, against its numpy float32 restatement fed the same per-step hits
  and tests: bit for bit;
* updateProbabilisticResidency's object-level decisions (host side, like the reference) against
  their numpy restatement over a moving camera: the same resident set after every step;
* the ray-hit budget with the reference's ray-hit prior: keys and selection against the oracle.
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


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_object_tests_match_oracle(nb, orc, ctx, small_city):
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    rng = np.random.default_rng(4)
    evicted = np.nonzero(rng.random(sb.object_count) < 0.3)[0]
    for o in evicted:
        ctx.set_object_active(int(o), False)
    ctx.flush()
    ctx.count_object_tests(True)
    rays = np.concatenate([raysets.aimed_rays(sb, 20000, 3), raysets.random_rays(sb, 8000, 4)])
    hits = ctx.trace_closest(rays, count_hits=True)
    got = ctx.count_object_tests(True, read=True)
    root = np.ascontiguousarray(sb.instances["blas_root_index"], np.int32).copy()
    root[evicted] = -1
    os_ = orc.OracleScene(sb, blas_root=root)
    ref = os_.closest(rays)
    assert np.array_equal(np.ascontiguousarray(hits).view(np.int32), np.ascontiguousarray(ref).view(np.int32))
    t = np.where(ref["prim"] >= 0, ref["t"], np.float32(np.inf)).astype(np.float32)
    want = ores.object_tests(os_, rays, t)
    assert got.sum() > rays.shape[0] and (got[evicted] == 0).all()
    assert np.array_equal(got, want), np.nonzero(got != want)[0][:10]
    # rendering counts tests on every bounce's closest-hit segments
    ctx.render(nb.view_pinhole((0, 60, -180), (0, 0, 0), width=64, height=36, spp=1, max_depth=2, seed=1),
               count_hits=True)
    assert ctx.count_object_tests(False, read=True).sum() > 64 * 36
    assert ctx.status() == 0


def _orbit(nb, frame, n=12):
    ang = frame * 0.35
    return nb.view_pinhole((150 * np.sin(ang), 55 + 5 * np.cos(frame), -150 * np.cos(ang)), (0, 0, 0),
                           width=96, height=54, spp=2, max_depth=2, seed=frame)


def test_posterior_and_probabilistic_policy_match_oracle(nb, orc, ctx, small_city):
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    N = sb.object_count
    counts = sb.instances["primitive_count"].astype(np.int64)
    kw = dict(target_fraction=0.6, min_active=16, max_toggles=6000, camera_motion=0.3, state_cooldown=5)
    prm = nb.ResidencyParams.make(nb.POLICY_PROBABILISTIC, **kw)
    post = ores.ObjectPosterior(N)
    pol = ores.ProbabilisticOracle(counts)
    active = ctx.residency_flags().astype(bool)
    evicted_any = restored_any = False
    for frame in range(14):
        view = _orbit(nb, frame)
        ctx.render(view, count_hits=True)
        pol.decrement_cooldowns()
        ctx.residency_step(prm, view, toggles=True)
        dev = ctx.residency_posterior()
        feats, _ = ctx.residency_last()
        visible = feats[:, 2] > 0.5
        post.step(dev["hits"], dev["tests"], visible, active)
        for k in ("alpha", "beta", "probability", "variance", "mass"):
            assert np.array_equal(_bits(dev[k]), _bits(getattr(post, k))), (frame, k)
        assert np.array_equal(dev["idle"], post.idle)
        want_active, _ = pol.step(post, dev["tests"], visible, active, frame + 1, **kw)
        got = ctx.residency_flags().astype(bool)
        assert np.array_equal(got, want_active), (frame, np.nonzero(got != want_active)[0][:10])
        assert np.array_equal(_bits(ctx.residency_posterior()["exploration"]), _bits(post.exploration)), frame
        evicted_any |= bool((active & ~got).any())
        restored_any |= bool((~active & got).any())
        active = got
    assert frame > 0 and dev["tests"].sum() > 0 and evicted_any and restored_any
    # traversal follows the resident set
    root = np.ascontiguousarray(sb.instances["blas_root_index"], np.int32).copy()
    root[~active] = -1
    rays = raysets.aimed_rays(sb, 6000, 7)
    got = ctx.trace_closest(rays)
    ref = orc.OracleScene(sb, blas_root=root).closest(rays)
    assert np.array_equal(np.ascontiguousarray(got).view(np.int32), np.ascontiguousarray(ref).view(np.int32))
    assert ctx.status() == 0


def test_rayhit_budget_with_prior_matches_oracle(nb, orc, ctx, small_city):
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    N = sb.object_count
    nbytes = ctx.object_bytes()
    budget = int(0.4 * nbytes.sum())
    prm = nb.ResidencyParams.make(nb.POLICY_RAYHIT_BUDGET, budget_bytes=budget, camera_motion=0.5,
                                  memory_pressure=0.25, min_active=2, rayhit_prior_scale=0.5)
    post = ores.ObjectPosterior(N)
    score = np.zeros(N, np.float32)
    flags = ctx.residency_flags()
    for frame in range(6):
        view = _orbit(nb, frame)
        ctx.reset_object_hits()
        ctx.render(view, count_hits=True)
        ctx.residency_step(prm, view, toggles=True)
        dev = ctx.residency_posterior()
        feats, keys = ctx.residency_last()
        visible = feats[:, 2] > 0.5
        hits = dev["hits"]
        post.step(hits, dev["tests"], visible, flags.astype(bool))
        score = (score * np.float32(0.85) + hits.astype(np.float32)).astype(np.float32)
        want_keys = (ores.rayhit_keys(score, hits, visible, 0.25) * ores.rayhit_prior(post.probability, 0.5))
        assert np.array_equal(_bits(keys), _bits(want_keys.astype(np.float32))), frame
        reserve = ores.reserve_count(N, 0.02, 0.06, 0.5)
        want, _ = ores.select(keys, visible, nbytes, budget, reserve, 2, flags)
        got = ctx.residency_flags()
        assert np.array_equal(got, want), frame
        flags = got
    assert (post.probability != 0.5).any() and ctx.status() == 0


@pytest.mark.parametrize("predictive", [False, True])
def test_environment_policies_match_oracle(nb, orc, ctx, small_city, predictive):
    """updateEnvironmentHitResidency / updatePredictiveResidency over a moving camera against
    their numpy restatement, fed the device's per-step hits, tests and escape statistics."""
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    N = sb.object_count
    counts = sb.instances["primitive_count"].astype(np.int64)
    policy = nb.POLICY_PREDICTIVE if predictive else nb.POLICY_ENVIRONMENT_HIT
    kw = dict(target_fraction=0.25, min_active=16, max_toggles=3000, camera_motion=0.3, state_cooldown=5)
    prm = nb.ResidencyParams.make(policy, **kw)
    post = ores.ObjectPosterior(N)
    pol = ores.EnvironmentOracle(counts, predictive=predictive)
    score = np.zeros(N, np.float32)
    active = ctx.residency_flags().astype(bool)
    ctx.reset_render_stats()
    prev = np.zeros(4, np.uint64)
    changed = 0
    for frame in range(12):
        view = _orbit(nb, frame)
        ctx.render(view, count_hits=True)
        stats = ctx.render_stats()
        seg, esc = int(stats[0] - prev[0]), int(stats[1] - prev[1])
        prev = stats.copy()
        escape = np.float32(esc) / np.float32(max(seg, 1)) if seg > 0 else np.float32(0)
        pol.decrement_cooldowns()
        ctx.residency_step(prm, view, toggles=True)
        dev = ctx.residency_posterior()
        feats, _ = ctx.residency_last()
        visible = feats[:, 2] > 0.5
        post.step(dev["hits"], dev["tests"], visible, active)
        assert np.array_equal(_bits(dev["probability"]), _bits(post.probability)), frame
        score = (score * np.float32(0.85) + dev["hits"].astype(np.float32)).astype(np.float32)
        want, _ = pol.step(post, dev["tests"], score, visible, active, escape, **kw)
        got = ctx.residency_flags().astype(bool)
        assert np.array_equal(got, want), (frame, np.nonzero(got != want)[0][:10])
        changed += int((got != active).sum())
        active = got
    assert changed > 0 and ctx.status() == 0


def test_energy_policy_matches_oracle(nb, orc, ctx, small_city):
    """updateEnergyImportance over a moving camera against its numpy restatement, fed the device's
    posterior and the step's screen coverage (checked against a float64 restatement)."""
    from oracle import residency as ores

    _, sb = small_city
    ctx.upload(sb)
    N = sb.object_count
    kw = dict(target_fraction=0.7, min_active=16, max_toggles=6000, camera_motion=0.3, state_cooldown=3)
    prm = nb.ResidencyParams.make(nb.POLICY_ENERGY, **kw)
    post = ores.ObjectPosterior(N)
    pol = ores.EnergyOracle(sb)
    spheres = ores.object_spheres(sb)
    score = np.zeros(N, np.float32)
    active = ctx.residency_flags().astype(bool)
    changed = 0
    for frame in range(12):
        view = _orbit(nb, frame)
        ctx.render(view, count_hits=True)
        pol.decrement_cooldowns()
        ctx.residency_step(prm, view, toggles=True)
        dev = ctx.residency_posterior()
        feats, _ = ctx.residency_last()
        post.step(dev["hits"], dev["tests"], feats[:, 2] > 0.5, active)
        score = (score * np.float32(0.85) + dev["hits"].astype(np.float32)).astype(np.float32)
        cov, in_view, _ = ctx.residency_object_state()
        c64, margin = ores.coverage_f64(spheres, view)
        assert ((np.abs(cov.astype(np.float64) - c64) <= 1e-3 * np.maximum(1.0, c64)) | (margin < 1e-4)).all(), frame
        want, _ = pol.step(post, score, cov, in_view.astype(bool), active, frame + 1, 96, 54, **kw)
        got = ctx.residency_flags().astype(bool)
        assert np.array_equal(got, want), (frame, np.nonzero(got != want)[0][:10])
        changed += int((got != active).sum())
        active = got
    assert changed > 0 and ctx.status() == 0
