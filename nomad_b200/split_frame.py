"""A frame split over ranks by rows, one process per GPU, each with a full scene replica.

Rank r of N renders rows [H*r//N, H*(r+1)//N) of every view through nomad_render_tiles (the
reference renders a frame as tiles of one view, TileDispatchRegion, Renderer.cpp:1261-1266 and
:7319-7581). A tile's paths are the view's own paths, so the bands put together equal the frame
one GPU renders, bit for bit. The two exchanges of a split frame are the radiance bands, which an
all-gather puts together on every rank, and the per-object hit counts, which
`hit_exchange.allreduce_object_hits` sums so that the residency step decides the same on every
rank; the sum of the bands' counts is the whole frame's. Geometry and rays never cross.

With the NCCL backend the bands stay on the device (one all-gather of equal-sized, row-padded
buffers over NVLink) and the frame is returned as a CUDA tensor; with any other backend (gloo)
they go through host memory and the frame is a numpy array.
"""
from __future__ import annotations

import numpy as np

from .hit_exchange import allreduce_object_hits


def row_bands(height: int, world: int) -> list[tuple[int, int]]:
    """(first row, row count) of each rank's band: contiguous, disjoint, covering all rows, sizes
    differing by at most one."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    return [(height * r // world, height * (r + 1) // world - height * r // world) for r in range(world)]


def band_tiles(views, rank: int, world: int) -> np.ndarray:
    """This rank's tile of every view: (origin_x, origin_y, width, height) rows."""
    tiles = []
    for v in views:
        w, h = int(v["width"]), int(v["height"])
        if h < world:
            raise ValueError(f"a view of {h} rows cannot give each of {world} ranks a band")
        y0, rows = row_bands(h, world)[rank]
        tiles.append((0, y0, w, rows))
    return np.asarray(tiles, np.uint32)


def render_split(ctx, views, group=None, count_hits: bool = False, graph: bool = True):
    """Renders `views` (nomad_view records) with this rank's row band of each and returns the
    whole frame on every rank: one (height, width, 3) image per view, CUDA tensors with NCCL,
    numpy arrays otherwise. With count_hits the per-object counts of all ranks are summed into
    every rank's counters afterwards (allreduce_object_hits)."""
    import torch
    import torch.distributed as dist

    from .native import VIEW_DTYPE

    views = np.ascontiguousarray(views, VIEW_DTYPE).reshape(-1)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    tiles = band_tiles(views, rank, world)
    # every rank sends the same number of floats: each band padded to the largest band's rows
    pad = [(int(v["height"]) + world - 1) // world * int(v["width"]) * 3 for v in views]
    mine = [int(t[2]) * int(t[3]) * 3 for t in tiles]
    per_rank = sum(pad)
    nccl = dist.get_backend(group) == "nccl"
    if nccl:
        rendered = torch.empty(sum(mine), dtype=torch.float32, device="cuda")
        ctx.render_tiles_dev(views, tiles, rendered.data_ptr(), count_hits=count_hits, graph=graph)
        ctx.sync()
        send = torch.zeros(per_rank, dtype=torch.float32, device="cuda")
    else:
        rendered = torch.from_numpy(np.concatenate(
            [im.reshape(-1) for im in ctx.render_tiles(views, tiles, count_hits=count_hits, graph=graph)]))
        send = torch.zeros(per_rank, dtype=torch.float32)
    so = ro = 0
    for p, m in zip(pad, mine):
        send[so:so + m] = rendered[ro:ro + m]
        so += p
        ro += m
    recv = torch.empty(world * per_rank, dtype=torch.float32, device=send.device)
    dist.all_gather_into_tensor(recv, send, group=group)
    frames = []
    off = 0
    for i, v in enumerate(views):
        w, h = int(v["width"]), int(v["height"])
        parts = []
        for r, (_, rows) in enumerate(row_bands(h, world)):
            base = r * per_rank + off
            parts.append(recv[base:base + rows * w * 3])
        img = torch.cat(parts).reshape(h, w, 3)
        frames.append(img if nccl else img.numpy())
        off += pad[i]
    if count_hits:
        allreduce_object_hits(ctx, group)
    return frames
