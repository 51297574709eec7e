"""Failure detection without a GPU fault: a bounded device wait that runs out reports it in the
status word, and the context keeps working.

The self-test entry point waits on a shared-memory mbarrier with the same bounded-poll helper as
the traversal's staged-node copy. Nothing completes the barrier in the failing case (no copy is
started, so nothing is left in flight); the kernel sets the status bit and returns.
"""
import numpy as np
import pytest

from tests import raysets

pytestmark = pytest.mark.gpu

WAIT_EXPIRED = 1 << 1


def test_bounded_wait_runs_out_and_reports(nb, orc, ico_scene):
    _, sb = ico_scene
    ctx = nb.Context(0)
    try:
        ctx.upload(sb)
        assert ctx.status() == 0
        ctx.selftest_bounded_wait(complete=True)
        assert ctx.status() == 0                      # the barrier completed: no expiry
        ctx.selftest_bounded_wait(complete=False)
        assert ctx.status() & WAIT_EXPIRED            # nothing completed it: the wait ran out
        assert ctx.status() == 0                      # reading cleared the word
        for _ in range(3):                            # repeatable, and nothing is left behind
            ctx.selftest_bounded_wait(complete=False)
        assert ctx.status() == WAIT_EXPIRED
        rays = np.concatenate([raysets.aimed_rays(sb, 5000, 3), raysets.random_rays(sb, 5000, 4)])
        got = ctx.trace_closest(rays)                 # the context still traces correctly
        want = orc.OracleScene(sb).closest(rays)
        assert np.array_equal(np.ascontiguousarray(got).view(np.int32), np.ascontiguousarray(want).view(np.int32))
        assert ctx.status() == 0
    finally:
        ctx.close()
