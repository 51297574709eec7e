"""Known-answer cases for the ray-hit budget policy, derived by hand from the reference's
updateRayHitBudget (Nomad Path Tracer/Renderer/RendererResidency.cpp:2755-2964), the per-frame
cooldown decrement of updateResidency (:205-207) and setPrimitiveActive's cooldown
(Renderer.cpp:7838-7839); in the pattern of the reference's own residency harness tests
(tests/ProbabilisticResidencyTests.cpp). Each case states the reference lines it follows and the
arithmetic of its expected answer.

They check the oracle's restatements (oracle/residency.py): RayHitPrimOracle, which the device
policy NOMAD_POLICY_RAYHIT_PRIM equals frame by frame on B200 (tests/test_residency_gpu.py), and the
per-object selection with its visibility reserve and byte budget used by NOMAD_POLICY_RAYHIT_BUDGET.
"""
import numpy as np

from oracle import residency as ores


def _step(o, hits, visible, **kw):
    return o.step(np.asarray(hits, np.uint32), np.asarray(visible, np.uint8), **kw)


def test_target_fraction_clamp_and_ceil():
    """:2776-2779 fraction = clamp(0.54 + 0.10 motion - 0.24 pressure, 0.34, 0.92);
    :2885-2888 targetActive = ceil(N * fraction), at least min_active, at most N.
    N = 10, scores 10..1 for primitives 0..9, all visible, min_active 2:
      motion 1: fraction 0.64, target ceil(6.4) = 7 -> primitives 7, 8, 9 evicted;
      pressure 1: fraction max(0.30, 0.34) = 0.34, target ceil(3.4) = 4 -> 4..9 evicted."""
    hits = np.arange(10, 0, -1)
    o = ores.RayHitPrimOracle(10)
    t = _step(o, hits, np.ones(10), motion=1.0, min_active=2)
    assert t == 3 and o.active.tolist() == [1] * 7 + [0] * 3
    o = ores.RayHitPrimOracle(10)
    t = _step(o, hits, np.ones(10), pressure=1.0, min_active=2, max_toggles=16)
    assert t == 6 and o.active.tolist() == [1] * 4 + [0] * 6


def test_equal_scores_keep_the_lower_index():
    """:2893-2899 the sort breaks equal scores by the lower index. N = 6, every primitive one hit
    and visible: target ceil(6 * 0.54) = ceil(3.24) = 4 -> primitives 0..3 stay, 4 and 5 leave."""
    o = ores.RayHitPrimOracle(6)
    t = _step(o, np.ones(6), np.ones(6), min_active=1)
    assert t == 2 and o.active.tolist() == [1, 1, 1, 1, 0, 0]


def test_offscreen_scores():
    """:2833-2840 off-screen without hits -> 0; off-screen with hits -> score * lerp(0.5, 0.2,
    pressure); visible without score -> 1. N = 4, visible [1, 0, 0, 1], hits [0, 5, 0, 3],
    pressure 0: adjusted [1, 2.5, 0, 3], order 3, 1, 0, 2; target ceil(4 * 0.54) = 3 -> primitive
    2 leaves. With pressure 1 the fraction is 0.34, target ceil(1.36) = 2, and primitive 1 keeps
    5 * 0.2 = 1 (ties primitive 0, lower index first): order 3, 0, 1, 2 -> 3 and 0 stay."""
    o = ores.RayHitPrimOracle(4)
    assert _step(o, [0, 5, 0, 3], [1, 0, 0, 1], min_active=1) == 1
    assert o.active.tolist() == [1, 1, 0, 1]
    o = ores.RayHitPrimOracle(4)
    assert _step(o, [0, 5, 0, 3], [1, 0, 0, 1], pressure=1.0, min_active=1) == 2
    assert o.active.tolist() == [1, 0, 0, 1]


def test_visibility_reserve():
    """:2906-2923 the first ceil(N * (0.02 + 0.06 motion)) visible primitives in score order are
    wanted beyond the target. N = 50, motion 0.5: fraction 0.59, target ceil(29.5) = 30; reserve
    ceil(2.5) = 3. Scores 50..1 for primitives 0..49; only 40..49 visible: 40, 41, 42 join the
    top 30, 17 leave (the budget llround(16 * 1.225) = 20 allows all)."""
    vis = np.zeros(50)
    vis[40:] = 1
    o = ores.RayHitPrimOracle(50)
    t = _step(o, np.arange(50, 0, -1), vis, motion=0.5, min_active=1)
    want = np.zeros(50, np.uint8)
    want[:30] = 1
    want[40:43] = 1
    assert t == 17 and np.array_equal(o.active, want)


def test_toggle_budget_in_index_order():
    """:2780-2786 budget = llround(16 * (1 + 0.45 motion + 0.6 pressure)); :2930-2946 toggles in
    primitive index order, stopping at the budget. N = 100, scores 1..100 for primitives 0..99 (the
    highest index scores most), target ceil(54) = 54: primitives 0..45 are unwanted, and only the
    first 16 of them (0..15) leave in this step."""
    o = ores.RayHitPrimOracle(100)
    t = _step(o, np.arange(1, 101), np.ones(100), min_active=1)
    want = np.ones(100, np.uint8)
    want[:16] = 0
    assert t == 16 and np.array_equal(o.active, want)


def test_cooldowns_and_rebuild_cooldown():
    """:2795-2802 after a step that changed residency, the next rayHitRebuildCooldownFrames steps do
    nothing; :2934-2936 a primitive toggled less than stateCooldownFrames steps ago keeps its state
    (Renderer.cpp:7838-7839 sets the cooldown, :205-207 counts it down once per step).
    N = 10, scores 10..1 (motion 1: target 7): step 1 evicts 7, 8, 9 and starts both cooldowns.
    With rebuild cooldown 4, steps 2..5 change nothing whatever the hits. With rebuild cooldown 0,
    step 2 wants 7, 8, 9 back (they now score 1000, so 4, 5, 6 fall out of the top 7): 4, 5, 6
    leave, but the cooldown of 7, 8, 9 (5, counted down to 4) blocks them; steps 3..5 change
    nothing; in step 6 their cooldown is 0 and they come back (4, 5, 6 are still cooling)."""
    hits = np.arange(10, 0, -1)
    back = np.concatenate([np.zeros(7), np.full(3, 1000)])
    o = ores.RayHitPrimOracle(10)
    assert _step(o, hits, np.ones(10), motion=1.0, min_active=1) == 3
    for _ in range(4):
        assert _step(o, back, np.ones(10), motion=1.0, min_active=1) == 0
        assert o.active.tolist() == [1] * 7 + [0] * 3
    assert _step(o, back, np.ones(10), motion=1.0, min_active=1) > 0
    o = ores.RayHitPrimOracle(10)
    kw = dict(motion=1.0, min_active=1, rebuild_cooldown=0)
    assert _step(o, hits, np.ones(10), **kw) == 3
    assert _step(o, back, np.ones(10), **kw) == 3
    assert o.active.tolist() == [1] * 4 + [0] * 6 and o.cooldown[7:].tolist() == [4] * 3
    for step in range(3, 6):
        assert _step(o, back, np.ones(10), **kw) == 0, step
        assert o.cooldown[7:].tolist() == [6 - step] * 3
    assert _step(o, back, np.ones(10), **kw) == 3
    assert o.active.tolist() == [1] * 4 + [0] * 3 + [1] * 3


def test_object_selection_byte_budget():
    """The per-object restatement (NOMAD_POLICY_RAYHIT_BUDGET): min_active highest keys first, then
    the visibility reserve, then the rest greedily in key order (ties to the lower index), an
    object that does not fit the byte budget skipped and the walk continued; toggles in index
    order up to max_toggles. Keys [5, 4, 4, 3, 2, 1], bytes [60, 30, 50, 20, 10, 10], budget 100,
    visible only object 5, reserve 1, min_active 1:
      min_active: object 0 (60 B);  reserve: object 5 (70 B);  then 1 (100 B), 2 no (150),
      3 no (120), 4 no (110) -> wanted {0, 1, 5}."""
    keys = np.array([5, 4, 4, 3, 2, 1], np.float32)
    nbytes = np.array([60, 30, 50, 20, 10, 10])
    vis = np.array([0, 0, 0, 0, 0, 1], bool)
    res, t = ores.select(keys, vis, nbytes, 100, 1, 1, np.ones(6, np.uint8))
    assert res.tolist() == [1, 1, 0, 0, 0, 1] and t == 3
    res, t = ores.select(keys, vis, nbytes, 100, 1, 1, np.ones(6, np.uint8), max_toggles=2)
    assert res.tolist() == [1, 1, 0, 0, 1, 1] and t == 2


def test_posterior_known_answers():
    """processRayHitCounters' object posterior (Renderer.cpp:8420-8522), from Beta(1, 1) with
    decay 0.9, evidence window 64, threshold 0.5, hit decay 0.85:
      3 hits of 5 tested: alpha 0.9 + 3 = 3.9, beta 0.9 + 2 = 2.9, p = 3.9 / 6.8, exploration
        0 (p >= 0.5: 0 * 0.85);
      0 hits of 2 tested: alpha 0.9, beta 2.9, p = 0.9 / (0.9 + 2.9) < 0.5 -> exploration 0 + 2 = 2;
      nothing tested (cooling, :8453-8477): alpha = beta = 0.9, p 0.5 cooled to 0.45 at mass 1.8
        -> alpha 0.81, beta 0.99; a visible or resident object seeds exploration 1, idle 1;
      1000 hits of 1000 tested: mass 1000.9 clamped to the window 64 (:8199-8214),
        alpha = 1000.9 * 64 / 1000.9, beta 0.9 * 64 / 1000.9."""
    f = np.float32
    p = ores.ObjectPosterior(5)
    p.step(np.array([3, 0, 0, 0, 1000], np.uint32), np.array([5, 2, 0, 0, 1000], np.uint32),
           [0, 0, 1, 0, 0], [0, 0, 0, 0, 0])
    assert p.alpha[0] == f(3.9) and p.beta[0] == f(2.9) and p.probability[0] == f(3.9) / f(6.8)
    a1, b1 = f(0.9) + f(0), f(0.9) + f(2)
    assert p.exploration[0] == 0 and p.exploration[1] == f(2) and p.probability[1] == a1 / (a1 + b1)
    assert p.alpha[2] == f(0.45) * f(1.8) and p.beta[2] == f(1.8) - f(0.45) * f(1.8)
    assert p.exploration[2] == 1 and p.exploration[3] == 0 and p.idle.tolist() == [0, 0, 1, 1, 0]
    s = f(1000.9)
    assert p.mass[4] == f(64) and p.alpha[4] == s * (f(64) / (s + f(0.9)))
    assert p.beta[4] == f(0.9) * (f(64) / (s + f(0.9)))


def test_resident_key_bonus():
    """The selection's hysteresis (no reference counterpart): a resident object's key k becomes
    k + bonus * |k|. Keys [5, 4.5, 4, 1], 10 bytes each, budget 20, objects 1 and 2 resident, no
    reserve: without a bonus objects 0 and 1 are wanted; with bonus 0.3 the resident keys become
    5.85 and 5.2, both above 5, so 1 and 2 stay and 0 is not brought in."""
    keys = np.array([5, 4.5, 4, 1], np.float32)
    nbytes = np.full(4, 10)
    vis = np.zeros(4, bool)
    cur = np.array([0, 1, 1, 0], np.uint8)
    res, t = ores.select(keys, vis, nbytes, 20, 0, 0, cur)
    assert res.tolist() == [1, 1, 0, 0] and t == 2
    res, t = ores.select(keys, vis, nbytes, 20, 0, 0, cur, resident_bonus=0.3)
    assert res.tolist() == [0, 1, 1, 0] and t == 0
