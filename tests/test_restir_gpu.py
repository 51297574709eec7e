"""ReSTIR DI: GPU passes against the scalar oracle over consecutive frames (temporal reuse), and
the estimator's error against a high-spp path-traced reference compared with one-sample NEE."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lit_city(nb):
    scene = nb.synth_city(seed=21, grid=8, size_m=250.0, target_tris=100_000, median_tris=800,
                          max_tris=15_000, emissive_quads=8, emissive_tris=512, emissive_sigma=1.5)
    return scene, nb.SceneBVH(scene)


@pytest.fixture(scope="module")
def ctx(nb):
    c = nb.Context(0)
    yield c
    c.close()


def test_restir_parity_two_frames(nb, orc, ctx, lit_city):
    scene, sb = lit_city
    ctx.upload(sb)
    ctx.set_restir(candidates=32, temporal=True, spatial=3, radius_px=30.0, m_cap=20.0)
    ctx.reset_render_stats()
    ref = orc.RestirOracle(orc.OracleScene(sb), sb.materials)
    for f, pos in enumerate([(0, 60, -180), (1.5, 60, -178.5), (3.0, 59.5, -177)]):
        v = np.concatenate([
            nb.view_pinhole(pos, (0, 10, 0), width=64, height=40, spp=2, max_depth=2, seed=3, frame=f,
                            flags=nb.VIEW_RESTIR),
            nb.view_pinhole((80, 30, 20), (0, 5, 0), width=24, height=16, spp=1, max_depth=3, seed=4, frame=f,
                            flags=nb.VIEW_RESTIR)])
        imgs = ctx.render(v)
        got = np.concatenate([i.reshape(-1, 3) for i in imgs])
        want, stats = ref.render(v)
        exact = (got == want).all(1).mean()
        err = (np.abs(got - want).sum(1) / np.maximum(np.abs(want).sum(1), 1e-6)).mean()
        assert err < 1e-4 and exact > 0.99, (f, err, exact)
    assert ctx.status() == 0


@pytest.mark.parametrize("graph", [True, False])
def test_restir_reference_mode_parity(nb, orc, ctx, lit_city, graph):
    """The reference's own ReSTIR (per-candidate visibility, previous-frame temporal and +-1 px
    spatial reuse with its MIS weights and Jacobian) against the oracle's restatement, over
    consecutive frames of a moving camera."""
    scene, sb = lit_city
    ctx.upload(sb)
    ctx.set_restir(candidates=24, temporal=True, reference_mode=True)
    ctx.reset_render_stats()
    ref = orc.RestirOracle(orc.OracleScene(sb), sb.materials, candidates=24, temporal=True, reference_mode=True)
    shadow = 0
    for f, pos in enumerate([(0, 60, -180), (1.0, 60, -179), (2.0, 59.8, -178), (3.0, 59.5, -177)]):
        v = np.concatenate([
            nb.view_pinhole(pos, (0, 10, 0), width=64, height=40, spp=1, max_depth=2, seed=3, frame=f,
                            flags=nb.VIEW_RESTIR),
            nb.view_pinhole((80, 30, 20), (0, 5, 0), width=24, height=16, spp=2, max_depth=3, seed=4, frame=f,
                            flags=nb.VIEW_RESTIR)])
        imgs = ctx.render(v, graph=graph)
        got = np.concatenate([i.reshape(-1, 3) for i in imgs])
        want, stats = ref.render(v)
        shadow += int(stats[2])
        exact = (got == want).all(1).mean()
        err = (np.abs(got - want).sum(1) / np.maximum(np.abs(want).sum(1), 1e-6)).mean()
        assert np.isfinite(got).all()
        assert err < 1e-4 and exact > 0.99, (f, err, exact)
    assert ctx.status() == 0
    # every candidate and reuse visibility ray is counted with the path's shadow rays
    assert ctx.render_stats()[2] == shadow


def test_restir_reduces_error(nb, ctx, lit_city):
    scene, sb = lit_city
    ctx.upload(sb)
    ctx.set_restir(candidates=32, temporal=True, spatial=3, radius_px=30.0, m_cap=20.0)
    pos, look = (0, 60, -180), (0, 10, 0)
    # direct lighting only (one bounce) through pixel centres, so NEE and ReSTIR estimate the same
    # quantity and the error is the light-sampling variance alone
    ref = ctx.render(nb.view_pinhole(pos, look, width=96, height=60, spp=1024, max_depth=1, seed=99,
                                     flags=nb.VIEW_CENTER))[0]
    errs = {"nee": [], "restir": []}
    ctx.reset_restir()
    for f in range(4):
        for name, flags in (("nee", 0), ("restir", nb.VIEW_RESTIR)):
            img = ctx.render(nb.view_pinhole(pos, look, width=96, height=60, spp=1, max_depth=1, seed=7, frame=f,
                                             flags=flags | nb.VIEW_CENTER))[0]
            errs[name].append(float(((img - ref) ** 2).mean() / (ref ** 2).mean()))
    nee, rst = np.mean(errs["nee"][1:]), np.mean(errs["restir"][1:])
    assert rst < 0.7 * nee, errs
