"""Tiles of a view (nomad_render_tiles) against the whole frame (nomad_render_frame).

A tile's paths are the view's own paths, so every tile pixel must equal that pixel of the whole
frame bit for bit (jittered camera rays, three bounces, NEE), and the per-object counts of tiles
that cover a view once must add up to the whole frame's. The whole frame is itself checked
against the oracle in test_pathtrace_gpu.py. Row bands as nomad_b200.split_frame hands them to
the ranks of a split frame, interior tiles of a two-view batch, device output, graph replays with
moved tiles, and the refused tiles are covered.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _view(nb, pos, w, h, seed, spp=2, depth=3, flags=0):
    v = nb.view_pinhole(pos, (0, 0, 0), width=w, height=h, spp=spp, max_depth=depth, seed=seed, frame=3)
    v["flags"] |= flags
    return v


@pytest.fixture(scope="module")
def cctx(nb, small_city):
    _, sb = small_city
    c = nb.Context(0)
    c.upload(sb)
    yield c
    c.close()


def test_row_bands_equal_the_frame(nb, cctx):
    from nomad_b200.split_frame import band_tiles

    v = _view(nb, (0, 60, -180), 160, 91, 7)
    cctx.reset_object_hits()
    whole = cctx.render(v, count_hits=True)[0]
    want_hits = cctx.object_hits().copy()
    assert want_hits.sum() > 0 and np.abs(whole).sum() > 0
    for world in (2, 3):
        cctx.reset_object_hits()
        bands = []
        for rank in range(world):
            t = band_tiles(v, rank, world)
            bands.append(cctx.render_tiles(v, t, count_hits=True)[0])
        assert np.array_equal(_bits(np.concatenate(bands)), _bits(whole)), world
        assert np.array_equal(cctx.object_hits(), want_hits), world


def test_interior_tiles_of_a_batch(nb, cctx):
    import torch

    views = np.concatenate([_view(nb, (0, 60, -180), 120, 70, 1), _view(nb, (40, 45, -120), 96, 54, 2, spp=3)])
    whole = cctx.render(views)
    tiles = [(37, 11, 50, 23), (0, 53, 7, 1)]
    got = cctx.render_tiles(views, tiles)
    for img, full, (x, y, w, h) in zip(got, whole, tiles):
        assert img.shape == (h, w, 3)
        assert np.array_equal(_bits(img), _bits(full[y:y + h, x:x + w]))
    # the same tiles into device memory
    out = torch.empty((50 * 23 + 7) * 3, dtype=torch.float32, device="cuda")
    cctx.render_tiles_dev(views, tiles, out.data_ptr())
    cctx.sync()
    dev = out.cpu().numpy()
    assert np.array_equal(_bits(dev), _bits(np.concatenate([g.reshape(-1) for g in got])))


def test_graph_replays_with_moved_tiles(nb, cctx):
    """Tiles of one shape at other origins replay the captured frame: the origins are read from
    the device view table, not baked into the graph."""
    v = _view(nb, (0, 60, -180), 128, 64, 9)
    whole = cctx.render(v, graph=False)[0]
    before = cctx.frame_graph_stats()
    for x, y in ((0, 0), (64, 0), (21, 40), (64, 32)):
        img = cctx.render_tiles(v, [(x, y, 64, 24)])[0]
        assert np.array_equal(_bits(img), _bits(whole[y:y + 24, x:x + 64])), (x, y)
    after = cctx.frame_graph_stats()
    assert after["captures"] - before["captures"] == 1
    assert after["launches"] - before["launches"] == 4


def test_refused_tiles(nb, cctx):
    v = _view(nb, (0, 60, -180), 64, 32, 1)
    for bad in ((0, 0, 0, 8), (0, 0, 8, 0), (60, 0, 5, 4), (0, 30, 8, 3), (64, 0, 1, 1)):
        with pytest.raises(nb.NomadError):
            cctx.render_tiles(v, [bad])
    with pytest.raises(ValueError):
        cctx.render_tiles(np.concatenate([v, v]), [(0, 0, 8, 8)])
    r = _view(nb, (0, 60, -180), 64, 32, 1, depth=1, flags=nb.VIEW_RESTIR)
    with pytest.raises(nb.NomadError, match="ReSTIR"):
        cctx.render_tiles(r, [(0, 0, 64, 16)])
    # the context stays usable
    img = cctx.render_tiles(v, [(0, 0, 64, 32)])[0]
    assert np.array_equal(_bits(img), _bits(cctx.render(v)[0]))


def test_nccl_single_rank_split_frame(nb, small_city):
    """The NCCL paths of render_split (device bands, row padding, all-gather) and of
    allreduce_object_hits (device counts, all-reduce, write-back) in a one-rank group, which one
    GPU can run: the frames equal the whole render bit for bit and the counts are kept."""
    import datetime
    import socket

    import torch.distributed as dist

    from nomad_b200.hit_exchange import allreduce_object_hits
    from nomad_b200.split_frame import render_split

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    c = nb.Context(0)
    try:
        c.upload(small_city[1])
        views = np.concatenate([_view(nb, (0, 60, -180), 120, 71, 4), _view(nb, (40, 45, -120), 96, 54, 5)])
        c.reset_object_hits()
        want = c.render(views, count_hits=True)
        want_hits = c.object_hits().copy()
        c.reset_object_hits()
        got = render_split(c, views, count_hits=True)
        assert len(got) == 2
        for g, w in zip(got, want):
            assert g.is_cuda and tuple(g.shape) == w.shape
            assert np.array_equal(_bits(g.cpu().numpy()), _bits(w))
        assert np.array_equal(c.object_hits(), want_hits)
        assert allreduce_object_hits(c) is None
        assert np.array_equal(c.object_hits(), want_hits)
    finally:
        c.close()
        dist.destroy_process_group()
