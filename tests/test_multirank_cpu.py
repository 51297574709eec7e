"""The multi-rank host logic of bench.py, on CPU with two `gloo` ranks.

bench.py runs one replica per GPU (the views shard; there is no data-path collective). What
crosses ranks is the timing: each rank's timed region is reduced to the slowest rank's
(`ranks_max`), and the whole-job throughput counts every rank's units (`job_rate`). The reference
arm does its work on rank 0 only; other ranks return at once. These are checked here with two
processes on 127.0.0.1; the GPU box has one GPU, so the NCCL run of the same code is not tested
on several GPUs.
"""
import os
import socket
import sys

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
