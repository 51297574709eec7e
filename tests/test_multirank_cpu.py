"""The multi-rank host logic of bench.py, on CPU with two `gloo` ranks.

bench.py runs one replica per GPU (the views shard; there is no data-path collective). What
crosses ranks is the timing: each rank's timed region is reduced to the slowest rank's
(`ranks_max`), and the whole-job throughput counts every rank's units (`job_rate`). The reference
arm does its work on rank 0 only; other ranks return at once. A frame split over ranks also sums
the per-object hit counters before the residency step (`nomad_b200.hit_exchange`). These are
checked here with two processes on 127.0.0.1; the GPU box has one GPU, so the NCCL run of the
same code is not tested on several GPUs.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import types

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = 10.0 + 7.5 * rank  # this rank's timed seconds
        slowest = bench.ranks_max(mine, world, device="cpu")
        dist.barrier()
        rate = bench.job_rate(world, 1_000_000, 4, slowest)
        # the reference arm: ranks other than 0 return without doing any work
        ref = bench.run_reference(types.SimpleNamespace(warmup=0, steps=1)) if rank != 0 else None
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{slowest!r} {rate!r} {ref!r}\n")
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_reduce_to_the_slowest(tmp_path):
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(world)]
    for slowest, rate, ref in rows:
        assert float(slowest) == 17.5                 # max over ranks, the same on every rank
        assert float(rate) == pytest.approx(2 * 1_000_000 * 4 / 17.5 / 1e6)
        assert ref == "None"


def test_single_rank_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.ranks_max(3.25, 1) == 3.25
    assert bench.job_rate(1, 8_000_000, 10, 2.0) == pytest.approx(40.0)


class _FakeCounters:
    """Stands in for a Context's per-object hit counters (host side only)."""

    def __init__(self, counts):
        self.object_count = len(counts)
        self.counts = np.asarray(counts, np.uint32)

    def object_hits(self):
        return self.counts.copy()

    def write_object_hits(self, counts=None, dev_ptr=0):
        assert not dev_ptr
        self.counts = np.asarray(counts, np.uint32).copy()


def _hits_rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    from nomad_b200.hit_exchange import allreduce_object_hits

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(100 + rank)  # each rank rendered its own views
        local = rng.integers(0, 3_000_000_000 // world, 2048, dtype=np.uint64).astype(np.uint32)
        np.save(os.path.join(out_dir, f"local{rank}.npy"), local)
        ctx = _FakeCounters(local)
        total = allreduce_object_hits(ctx)
        np.save(os.path.join(out_dir, f"total{rank}.npy"), ctx.counts)
        assert np.array_equal(total, ctx.counts)
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(180)
def test_two_gloo_ranks_sum_object_hits(tmp_path):
    """Two ranks that rendered different views end with the same, summed per-object counts
    (values above 2^31 included), which their residency steps then read."""
    world = 2
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_hits_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(150)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    want = sum(np.load(tmp_path / f"local{r}.npy").astype(np.uint64) for r in range(world))
    assert want.max() > 2**31
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"total{r}.npy"), want.astype(np.uint32))
