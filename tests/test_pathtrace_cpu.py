"""CPU tests of the oracle path tracer's building blocks."""
import ctypes

import numpy as np


def test_philox_known_answers(orc):
    """Random123's published known-answer vectors for Philox4x32-10."""
    lib = orc.load()
    kat = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
           ((0xffffffff,) * 4, (0xffffffff,) * 2, (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
           ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
            (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in kat:
        c = (ctypes.c_uint32 * 4)(*ctr)
        k = (ctypes.c_uint32 * 2)(*key)
        o = (ctypes.c_uint32 * 4)()
        lib.oracle_philox(c, k, o)
        assert tuple(o) == want


def test_math_polynomials(orc):
    """The fixed sin/cos/log2/exp2 definitions stay within 1e-6 of the true functions."""
    lib = orc.load()
    o = (ctypes.c_float * 4)()
    worst = np.zeros(4)
    for u in np.linspace(0.0, 0.999999, 4001, dtype=np.float32):
        lib.oracle_math(ctypes.c_float(u), o)
        ref = [np.sin(2 * np.pi * float(u)), np.cos(2 * np.pi * float(u)),
               np.log2(float(u)) if u > 0 else 0.0, 2.0 ** (-4.0 * float(u))]
        err = [abs(o[0] - ref[0]), abs(o[1] - ref[1]), abs(o[2] - ref[2]) / max(1.0, abs(ref[2])),
               abs(o[3] - ref[3]) / ref[3]]
        worst = np.maximum(worst, err)
    assert (worst < 2e-6).all(), worst


def test_oracle_render_converges(nb, orc, small_city):
    """Radiance estimates with independent seeds agree in expectation (sanity of the sampler)."""
    scene, sb = small_city
    os_ = orc.OracleScene(sb)
    means = []
    for seed in (1, 2):
        v = nb.view_pinhole((0, 60, -180), (0, 0, 0), width=32, height=18, spp=16, max_depth=3, seed=seed)
        rgb, _, st = orc.render(os_, sb.materials, v)
        assert np.isfinite(rgb).all() and (rgb >= 0).all()
        means.append(rgb.mean(0))
    assert np.allclose(means[0], means[1], rtol=0.05), means


def test_oracle_restir_reference_mode_reuses(nb, orc, small_city):
    """The oracle's restatement of the reference's ReSTIR: finite, non-negative radiance, and on
    the second frame the previous frame's reservoirs are reused (more visibility rays traced for
    the same candidates)."""
    _, sb = small_city
    ref = orc.RestirOracle(orc.OracleScene(sb), sb.materials, candidates=8, temporal=True, reference_mode=True)
    counts = []
    for f, pos in enumerate([(0, 60, -120), (0.5, 60, -119.5)]):
        v = nb.view_pinhole(pos, (0, 10, 0), width=24, height=16, spp=1, max_depth=1, seed=3, frame=f,
                            flags=nb.VIEW_RESTIR | nb.VIEW_CENTER)
        rgb, stats = ref.render(v)
        assert np.isfinite(rgb).all() and (rgb >= 0).all()
        counts.append(int(stats[2]))
    assert counts[1] > counts[0]
