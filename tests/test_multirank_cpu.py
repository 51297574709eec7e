"""The multi-rank host logic of bench.py, on CPU with two `gloo` ranks.

bench.py runs one replica per GPU (the views shard; there is no data-path collective). What
crosses ranks is the timing: each rank's timed region is reduced to the slowest rank's
(`ranks_max`), and the whole-job throughput counts every rank's units (`job_rate`). The reference
arm does its work on rank 0 only; other ranks return at once. A frame split over ranks also sums
the per-object hit counters before the residency step (`nomad_b200.hit_exchange`) and gathers the
row bands each rank rendered (`nomad_b200.split_frame`). These are
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


class _FakeTiles(_FakeCounters):
    """Stands in for a Context's tile rendering: a pixel's value depends only on its view and its
    place in the whole view, like the paths of nomad_render_tiles, and every rendered pixel
    counts one hit on object (pixel index mod object count)."""

    def __init__(self, objects):
        super().__init__(np.zeros(objects, np.uint32))

    def render_tiles(self, views, tiles, count_hits=False, graph=True):
        out = []
        for i, (v, (x0, y0, w, h)) in enumerate(zip(views, tiles)):
            W = int(v["width"])
            ys, xs = np.meshgrid(np.arange(y0, y0 + h), np.arange(x0, x0 + w), indexing="ij")
            pix = ys * W + xs
            img = np.stack([np.sin(pix * 0.37 + i + c).astype(np.float32) for c in range(3)], -1)
            out.append(img)
            if count_hits:
                np.add.at(self.counts, pix.reshape(-1) % self.object_count, 1)
        return out


def _views(dims):
    from nomad_b200.native import VIEW_DTYPE

    v = np.zeros(len(dims), VIEW_DTYPE)
    for i, (w, h) in enumerate(dims):
        v[i]["width"], v[i]["height"], v[i]["spp"], v[i]["max_depth"] = w, h, 1, 1
    return v


SPLIT_VIEWS = [(13, 7), (5, 11), (8, 3)]


def _split_rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    from nomad_b200.split_frame import render_split

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ctx = _FakeTiles(17)
        frames = render_split(ctx, _views(SPLIT_VIEWS), count_hits=True)
        for i, f in enumerate(frames):
            np.save(os.path.join(out_dir, f"frame{rank}_{i}.npy"), f)
        np.save(os.path.join(out_dir, f"hits{rank}.npy"), ctx.counts)
    finally:
        dist.barrier()
        dist.destroy_process_group()


@pytest.mark.timeout(240)
def test_three_gloo_ranks_split_a_frame_by_rows(tmp_path):
    """Three ranks render uneven row bands (7 rows: 2 + 2 + 3; 3 rows: one each) of three views;
    every rank ends with the whole frames, equal to one rank's render of the whole views, and
    with the whole frame's per-object counts."""
    world = 3
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_split_rank_main, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(200)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    whole = _FakeTiles(17)
    views = _views(SPLIT_VIEWS)
    want = whole.render_tiles(views, [(0, 0, w, h) for w, h in SPLIT_VIEWS], count_hits=True)
    for r in range(world):
        for i in range(len(SPLIT_VIEWS)):
            got = np.load(tmp_path / f"frame{r}_{i}.npy")
            assert got.shape == want[i].shape and np.array_equal(got, want[i]), (r, i)
        assert np.array_equal(np.load(tmp_path / f"hits{r}.npy"), whole.counts), r


def test_row_bands_partition_the_rows():
    from nomad_b200.split_frame import band_tiles, row_bands

    for h in (1, 2, 7, 1080, 1081):
        for world in (1, 2, 3, 8):
            bands = row_bands(h, world)
            assert len(bands) == world
            assert bands[0][0] == 0 and sum(b[1] for b in bands) == h
            assert all(bands[r][0] + bands[r][1] == bands[r + 1][0] for r in range(world - 1))
            assert max(b[1] for b in bands) - min(b[1] for b in bands) <= 1
    t = band_tiles(_views([(640, 360), (17, 9)]), 2, 4)
    assert t.tolist() == [[0, 180, 640, 90], [0, 4, 17, 2]]
    with pytest.raises(ValueError):
        band_tiles(_views([(640, 3)]), 0, 4)  # a band per rank needs at least as many rows
    with pytest.raises(ValueError):
        row_bands(10, 0)
