"""Host logic of the residency comparison (nomad_b200.residency_eval), without a GPU: the camera
path, the repeat/spread bookkeeping, the hits-per-byte targets, the fixed traversal, and the rules
that choose a budget or a paged configuration from a sweep and judge it against the ray-hit
policy."""
import numpy as np
import pytest

from nomad_b200 import residency_eval as rev


def test_catmull_rom_passes_through_the_control_points():
    pts = np.array([[0, 0, 0], [10, 5, 0], [20, 0, 10], [30, 5, 10]], np.float32)
    # 3 segments, 7 samples: every second sample lands on a control point
    out = rev.catmull_rom(pts, 7)
    assert out.shape == (7, 3) and out.dtype == np.float32
    np.testing.assert_allclose(out[::2], pts, atol=1e-5)
    # the midpoint of a straight, evenly spaced run is the segment's midpoint
    line = np.array([[0, 0, 0], [1, 0, 0], [2, 0, 0], [3, 0, 0]], np.float32)
    np.testing.assert_allclose(rev.catmull_rom(line, 7)[3], [1.5, 0, 0], atol=1e-6)


def test_camera_path_is_seeded_and_stays_over_the_city():
    a = rev.camera_path(3, 50, 2000.0, 1000.0)
    b = rev.camera_path(3, 50, 2000.0, 1000.0)
    c = rev.camera_path(4, 50, 2000.0, 1000.0)
    assert len(a) == 50
    assert all(np.array_equal(p, q) and np.array_equal(l, m) for (p, l), (q, m) in zip(a, b))
    assert not all(np.array_equal(p, q) for (p, _), (q, _) in zip(a, c))
    for pos, look in a:
        # positions inside the city's central 90 % (the spline overshoots its controls a little)
        assert abs(pos[0]) <= 0.5 * 2000.0 and abs(pos[2]) <= 0.5 * 1000.0
        d = look - pos
        # 60 m ahead on the ground plane, 25 m down
        assert d[1] == pytest.approx(-25.0, abs=1e-3)
        assert np.hypot(d[0], d[2]) == pytest.approx(60.0, rel=1e-4)


def test_repeat_reports_the_mean_and_spread_of_ms_per_frame():
    runs = iter([{"ms_per_frame": 2.0, "rel_mse_energy": 0.5, "x": 1},
                 {"ms_per_frame": 1.0, "rel_mse_energy": 0.5, "x": 2},
                 {"ms_per_frame": 3.0, "rel_mse_energy": 0.5, "x": 3}])
    out = rev.repeat(lambda: next(runs), 3)
    assert out["x"] == 1  # the first run's record
    assert out["ms_per_frame"] == pytest.approx(2.0)
    assert out["ms_per_frame_spread"] == {"mean": 2.0, "min": 1.0, "max": 3.0, "runs": [2.0, 1.0, 3.0]}
    assert out["rel_mse_energy_runs"] == [0.5, 0.5, 0.5] and out["repeats"] == 3


def test_cost_targets_weigh_hits_by_mean_size_over_size():
    kib = np.array([1.0, 4.0, 16.0, 64.0])
    hits = np.array([10.0, 10.0, 0.0, 100.0])
    x = np.zeros((4, 20), np.float32)
    x[:, 13] = np.log1p(kib)
    t = np.log1p(hits).astype(np.float32)
    got = rev.Workload.cost_targets(x, t)
    want = np.log1p(hits * kib.mean() / kib)
    np.testing.assert_allclose(got, want, rtol=1e-5)
    assert got.dtype == np.float32 and got[2] == 0.0


class _Ctx:
    def __init__(self):
        self.trav = None

    def set_traversal(self, **kw):
        self.trav = kw


def test_fix_traversal_sets_one_configuration_on_every_context():
    w = rev.Workload.__new__(rev.Workload)  # no scene: fix_traversal touches only the contexts
    a, b = _Ctx(), _Ctx()
    name = w.fix_traversal(a, b)
    assert a.trav == b.trav == rev.TRAVERSAL
    assert rev.TRAVERSAL["width"] == 4 and rev.TRAVERSAL["persistent"] == 1
    assert name == f"bvh{rev.TRAVERSAL['width']}_persist_mb{rev.TRAVERSAL['min_blocks']}"


def _rec(err, ms, lo=None, hi=None):
    r = {"rel_mse_energy": err, "ms_per_frame": ms}
    if lo is not None:
        r["ms_per_frame_spread"] = {"mean": ms, "min": lo, "max": hi, "runs": [lo, ms, hi]}
    return r


def test_smallest_budget_within_orders_budgets_numerically():
    sweep = {"0.10": _rec(0.9, 1.0), "0.15": _rec(0.30, 1.0), "0.20": _rec(0.20, 1.0), "0.35": _rec(0.1, 1.0)}
    assert rev.smallest_budget_within(sweep, 0.31) == "0.15"
    assert rev.smallest_budget_within(sweep, 0.2) == "0.20"
    assert rev.smallest_budget_within(sweep, 0.05) is None
    # an errored entry (no error figure) never qualifies
    assert rev.smallest_budget_within({"0.10": {"error": "x"}, "0.25": _rec(0.1, 1.0)}, 1.0) == "0.25"


def test_cheapest_within_takes_the_smallest_budget_then_the_lower_error():
    sweep = {"0.150/0.5": _rec(0.69, 1.20), "0.150/1": _rec(0.59, 1.21), "0.200/0.5": _rec(0.40, 1.10),
             "0.300/1": _rec(0.20, 1.40), "0.100/1": {"error": "pool too small"}}
    # both 15 % settings meet the bound: the lower error wins, whatever their ms/frame
    assert rev.cheapest_within(sweep, 0.79) == "0.150/1"
    assert rev.cheapest_within(sweep, 0.65) == "0.150/1"
    assert rev.cheapest_within(sweep, 0.5) == "0.200/0.5"
    assert rev.cheapest_within(sweep, 0.1) is None
    # the choice depends on budgets and errors only: other timings give the same key
    retimed = {k: (dict(v, ms_per_frame=2.0 - v["ms_per_frame"]) if "ms_per_frame" in v else v)
               for k, v in sweep.items()}
    assert rev.cheapest_within(retimed, 0.79) == "0.150/1"
    # budgets compare as numbers: 0.175 comes after 0.15
    assert rev.cheapest_within({"0.175/1": _rec(0.1, 1.0), "0.150/1": _rec(0.2, 1.0)}, 1.0) == "0.150/1"


def test_faster_outside_spread_and_within_5pct():
    rh = _rec(0.448, 1.32, 1.31, 1.33)
    assert rev.faster_outside_spread(_rec(0.3, 1.27, 1.26, 1.28), rh)
    assert not rev.faster_outside_spread(_rec(0.3, 1.30, 1.29, 1.315), rh)  # spreads overlap
    assert not rev.faster_outside_spread(_rec(0.3, 1.0), rh)  # no spread recorded
    assert rev.within_5pct(_rec(0.470, 1.0), rh)
    assert not rev.within_5pct(_rec(0.471, 1.0), rh)
    assert not rev.within_5pct({"error": "x"}, rh)
