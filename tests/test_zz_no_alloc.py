"""The allocation-free closest-hit entry point (nomad_trace_closest_noalloc).

It serves callers that cannot allocate GPU memory while tracing — a frame loop whose memory
budget is fully committed to resident geometry, or one that cannot take the implicit device
synchronisation of cudaMalloc/cudaFree mid-frame — by keeping its scratch in a static device
array. Its results must equal the regular entry point's (nomad_trace_closest with per-object
hit counting) and the oracle's: hits bit for bit, counts exactly. Two calls in a row check that
the shared scratch is cleared between calls. This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from tests import raysets

pytestmark = pytest.mark.gpu


def test_noalloc_matches_regular_entry_point(nb, orc):
    import torch

    scene = nb.synth_city(seed=5, grid=8, size_m=250.0, target_tris=120_000, median_tris=1000,
                          max_tris=20_000, emissive_quads=8)
    sb = nb.SceneBVH(scene)
    ctx = nb.Context(0)
    try:
        ctx.upload(sb)
        lib = ctx.lib
        for call, seed in enumerate((31, 32)):
            rays = np.concatenate([raysets.aimed_rays(sb, 30000, seed),
                                   raysets.random_rays(sb, 10000, seed + 100)])
            n = rays.shape[0]
            # regular entry point, host buffers, counters reset first
            ctx.reset_object_hits()
            want = ctx.trace_closest(rays, count_hits=True)
            want_counts = ctx.object_hits()
            # allocation-free entry point, device buffers owned by the caller
            d_rays = torch.from_numpy(rays.view(np.float32).reshape(-1, 8)).cuda()
            d_hits = torch.full((n, 5), -7, dtype=torch.int32, device="cuda")
            d_counts = torch.full((sb.object_count,), 12345, dtype=torch.int32, device="cuda")
            torch.cuda.synchronize()
            st = lib.nomad_trace_closest_noalloc(ctx.h, ctypes.c_void_p(d_rays.data_ptr()), n,
                                                 ctypes.c_void_p(d_hits.data_ptr()),
                                                 ctypes.c_void_p(d_counts.data_ptr()))
            assert st == 0, lib.nomad_last_error(ctx.h)
            ctx.sync()
            got = d_hits.cpu().numpy()
            assert np.array_equal(got, np.ascontiguousarray(want).view(np.int32).reshape(-1, 5)), \
                f"call {call}: hits differ"
            assert np.array_equal(d_counts.cpu().numpy().view(np.uint32), want_counts), \
                f"call {call}: per-object hit counts differ"
            assert want_counts.sum() == (want["prim"] >= 0).sum()
            # and both equal the oracle: its closest hits bit for bit, its per-object counts
            ref = orc.OracleScene(sb).closest(rays, orc.MODE_REFERENCE_ORDER)
            assert np.array_equal(got, np.ascontiguousarray(ref).view(np.int32).reshape(-1, 5)), \
                f"call {call}: hits differ from the oracle"
            ref_counts = np.bincount(ref["inst"][ref["prim"] >= 0], minlength=sb.object_count)
            assert np.array_equal(d_counts.cpu().numpy().view(np.uint32), ref_counts.astype(np.uint32)), \
                f"call {call}: per-object hit counts differ from the oracle's"
        assert ctx.status() == 0
    finally:
        ctx.close()
