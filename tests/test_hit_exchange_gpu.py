"""A frame split over ranks, emulated with two contexts on one GPU (the kernels of the two
"ranks" never wait on one another: they only exchange counts between launches).

Each context renders one of two views with hit counting on; the summed counts written back into
both (nomad_write_object_hits, from host memory and from device memory) make their residency
steps equal to that of a third context that rendered both views in one call. Primary rays only,
without jitter: a view's random streams depend on its index in the batch, so only then do the
split and the joint render trace the same rays.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _views(nb, frame):
    out = []
    for pos, w, h, seed in (((0, 60, -180), 96, 54, 1), ((40, 45, -120), 80, 60, 2)):
        v = nb.view_pinhole(pos, (0, 0, 0), width=w, height=h, spp=2, max_depth=1, seed=seed, frame=frame)
        v["flags"] |= nb.VIEW_CENTER
        out.append(v)
    return out


def test_split_frame_counts_and_residency(nb, small_city):
    import torch

    _, sb = small_city
    ctxs = [nb.Context(0) for _ in range(3)]
    try:
        for c in ctxs:
            c.upload(sb)
        nbytes = ctxs[0].object_bytes()
        prm = nb.ResidencyParams.make(nb.POLICY_RAYHIT_BUDGET, budget_bytes=int(0.4 * nbytes.sum()),
                                      camera_motion=0.5, min_active=2)
        a, b, joint = ctxs
        changed = False
        for frame in range(4):
            va, vb = _views(nb, frame)
            for c in ctxs:
                c.reset_object_hits()
            a.render(va, count_hits=True)
            b.render(vb, count_hits=True)
            joint.render(np.concatenate([va, vb]), count_hits=True)
            ha, hb, hj = a.object_hits(), b.object_hits(), joint.object_hits()
            total = ha.astype(np.uint64) + hb
            assert np.array_equal(total, hj) and hj.sum() > 0
            # rank a gets the sum from host memory, rank b from a device array
            a.write_object_hits(total.astype(np.uint32))
            d = torch.from_numpy(total.astype(np.int32)).cuda()
            torch.cuda.synchronize()
            b.write_object_hits(dev_ptr=d.data_ptr())
            b.sync()
            assert np.array_equal(a.object_hits(), hj) and np.array_equal(b.object_hits(), hj)
            out = torch.zeros(sb.object_count, dtype=torch.int32, device="cuda")
            b.object_hits_dev(out.data_ptr())
            b.sync()
            assert np.array_equal(out.cpu().numpy().astype(np.uint32), hj)
            for c in ctxs:
                c.residency_step(prm, va)
            fa, fb, fj = a.residency_flags(), b.residency_flags(), joint.residency_flags()
            assert np.array_equal(fa, fj) and np.array_equal(fb, fj), frame
            changed |= bool((fj == 0).any())
        assert changed  # the budget evicted something, so the equality says something
    finally:
        for c in ctxs:
            c.close()
