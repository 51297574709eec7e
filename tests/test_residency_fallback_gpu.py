"""The learned policy's fallback and the model file.

Without a usable model (none set yet, or the last nomad_mlp_set / nomad_mlp_load rejected), a
NOMAD_POLICY_LEARNED step runs the ray-hit budget step: frame for frame the same residency as a
context that runs NOMAD_POLICY_RAYHIT_BUDGET, with the fallback counted. A saved model loads back
bit for bit and scores like the original; damaged files (bad magic, version, size, checksum,
non-finite values) are refused with a reason and leave the context falling back.
"""
import struct

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _views(nb, frames):
    out = []
    for f in range(frames):
        ang = 0.35 * f
        out.append(nb.view_pinhole((160 * np.sin(ang), 60, -160 * np.cos(ang)), (0, 0, 0), width=96, height=54,
                                   spp=2, max_depth=2, seed=f))
    return out


def _run(nb, ctx, prm, views):
    flags, scores = [], []
    for v in views:
        ctx.reset_object_hits()
        ctx.render(v, count_hits=True)
        ctx.residency_step(prm, v)
        flags.append(ctx.residency_flags().copy())
        scores.append(ctx.residency_last()[1].copy())
    return flags, scores


def _fresh(nb, sb):
    c = nb.Context(0)
    c.upload(sb)
    return c


def _fnv1a(data: bytes) -> int:
    h = 1469598103934665603
    for b in data:
        h = ((h ^ b) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _model_file(blob, version=1, magic=b"NMLP", params=None, feats=24):
    params = blob.size if params is None else params
    body = magic + struct.pack("<III", version, params, feats) + np.asarray(blob, "<f4").tobytes()
    return body + struct.pack("<Q", _fnv1a(body))


def test_learned_without_model_runs_the_rayhit_budget(nb, small_city):
    _, sb = small_city
    views = _views(nb, 6)
    a, b = _fresh(nb, sb), _fresh(nb, sb)
    try:
        budget = int(a.object_bytes().sum() * 0.4)
        fa, sa = _run(nb, a, nb.ResidencyParams.make(nb.POLICY_LEARNED, budget_bytes=budget), views)
        fb, sb_ = _run(nb, b, nb.ResidencyParams.make(nb.POLICY_RAYHIT_BUDGET, budget_bytes=budget), views)
        for f in range(len(views)):
            assert np.array_equal(fa[f], fb[f]), f
            assert np.array_equal(sa[f].view(np.int32), sb_[f].view(np.int32)), f
        assert a.residency_fallback_steps() == len(views)
        assert b.residency_fallback_steps() == 0
        assert 0 < fa[-1].sum() < sb.object_count
    finally:
        a.close()
        b.close()


def test_model_file_round_trip(nb, small_city, tmp_path):
    _, sb = small_city
    views = _views(nb, 3)
    a, b = _fresh(nb, sb), _fresh(nb, sb)
    try:
        a.mlp_init(11)
        path = str(tmp_path / "model.nmlp")
        a.mlp_save(path)
        b.mlp_load(path)
        assert np.array_equal(a.mlp_get().view(np.int32), b.mlp_get().view(np.int32))
        budget = int(a.object_bytes().sum() * 0.4)
        prm = nb.ResidencyParams.make(nb.POLICY_LEARNED, budget_bytes=budget)
        fa, sa = _run(nb, a, prm, views)
        fb, sb_ = _run(nb, b, prm, views)
        for f in range(len(views)):
            assert np.array_equal(fa[f], fb[f]) and np.array_equal(sa[f].view(np.int32), sb_[f].view(np.int32))
        assert a.residency_fallback_steps() == 0 and b.residency_fallback_steps() == 0
    finally:
        a.close()
        b.close()


def test_damaged_model_files_are_refused_and_fall_back(nb, small_city, tmp_path):
    _, sb = small_city
    ctx = _fresh(nb, sb)
    try:
        ctx.mlp_init(5)
        good = ctx.mlp_get()
        path = tmp_path / "good.nmlp"
        ctx.mlp_save(str(path))
        raw = path.read_bytes()
        assert raw == _model_file(good)  # the documented layout, byte for byte
        nan_blob = good.copy()
        nan_blob[100] = np.nan
        flipped = bytearray(raw)
        flipped[40] ^= 0x01
        cases = {"magic": (_model_file(good, magic=b"XMLP"), "not a model file"),
                 "version": (_model_file(good, version=2), "format version 2"),
                 "shape": (_model_file(good[:-1], params=good.size - 1), "shape differs"),
                 "size": (raw[:-9], "size"),
                 "checksum": (bytes(flipped), "checksum mismatch"),
                 "nan": (_model_file(nan_blob), "not finite")}
        budget = int(ctx.object_bytes().sum() * 0.4)
        prm = nb.ResidencyParams.make(nb.POLICY_LEARNED, budget_bytes=budget)
        view = _views(nb, 1)[0]
        expected_fallbacks = 0
        for name, (data, why) in cases.items():
            ctx.mlp_load(str(path))  # a usable model again
            ctx.residency_step(prm, view)
            assert ctx.residency_fallback_steps() == expected_fallbacks, name
            bad = tmp_path / f"{name}.nmlp"
            bad.write_bytes(data)
            with pytest.raises(nb.NomadError, match=why):
                ctx.mlp_load(str(bad))
            ctx.residency_step(prm, view)
            expected_fallbacks += 1
            assert ctx.residency_fallback_steps() == expected_fallbacks, name
        with pytest.raises(nb.NomadError, match="cannot be opened"):
            ctx.mlp_load(str(tmp_path / "missing.nmlp"))
        ctx.mlp_set(good)
        with pytest.raises(nb.NomadError, match="not finite"):
            ctx.mlp_set(nan_blob)
        ctx.residency_step(prm, view)
        assert ctx.residency_fallback_steps() == expected_fallbacks + 1
    finally:
        ctx.close()
