"""GPU SceneBVH builder: the same arrays as the host builder (itself pinned to the reference's
Scene::buildBVH), bit for bit, on seeded scenes and on hand-made degenerate cases."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    for name in ("bvh_nodes", "tlas_nodes", "prims", "materials", "prim_indices", "object_bounds"):
        x, y = getattr(a, name), getattr(b, name)
        assert x.shape == y.shape, name
        assert np.array_equal(x.view(np.int32), y.view(np.int32)), name
    assert np.array_equal(a.instances.view(np.int32), b.instances.view(np.int32))
    assert a.max_depth == b.max_depth


def _edge_scene(nb, seed=3):
    """Objects with quantised coordinates (equal centroids, -0.0), spheres, rectangles, an object
    of identical triangles, a flat object, an empty object and a 30k-triangle object (radix path)."""
    rng = np.random.default_rng(seed)
    types, geoms, counts = [], [], []

    def add(t, g):
        types.append(np.asarray(t, np.int32))
        geoms.append(np.asarray(g, np.float32).reshape(-1, 15))
        counts.append(len(t))

    g = np.zeros((300, 15), np.float32)
    g[:, :9] = np.round(rng.uniform(-3, 3, (300, 9)))  # integers: ties and zeros
    g[::7, 0] = -0.0
    add(np.ones(300), g)
    g = np.zeros((120, 15), np.float32)
    g[:, :3] = rng.uniform(-50, 50, (120, 3))
    g[:, 3] = rng.uniform(0.1, 3, 120)
    add(np.zeros(120), g)
    g = np.zeros((90, 15), np.float32)
    g[:, :3] = rng.uniform(-20, 20, (90, 3))
    g[:, 3:6] = rng.uniform(-2, 2, (90, 3))
    g[:, 6:9] = rng.uniform(-2, 2, (90, 3))
    add(np.full(90, 2), g)
    g = np.zeros((40, 15), np.float32)
    g[:, :9] = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0], np.float32)
    add(np.ones(40), g)
    g = np.zeros((200, 15), np.float32)
    g[:, :9] = rng.uniform(-10, 10, (200, 9))
    g[:, [2, 5, 8]] = 0.0
    add(np.ones(200), g)
    add(np.zeros(0), np.zeros((0, 15)))
    g = np.zeros((30000, 15), np.float32)
    base = rng.uniform(-100, 100, (30000, 3)).astype(np.float32)
    g[:, 0:3] = base
    g[:, 3:6] = base + rng.uniform(-1, 1, (30000, 3))
    g[:, 6:9] = base + rng.uniform(-1, 1, (30000, 3))
    g[:, 9:15] = rng.uniform(0, 1, (30000, 6))
    add(np.ones(30000), g)
    t = np.concatenate(types)
    geo = np.concatenate(geoms)
    mat = np.zeros((t.shape[0], 20), np.float32)
    mat[:, 0:3] = 0.7
    mat[:, 3] = 1.0
    mat[:, 7] = 1.0
    first = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint32)
    return nb.HostScene(t, geo, mat, first, np.asarray(counts, np.uint32))


@pytest.mark.parametrize("which", ["edge", "ico", "city"])
def test_gpu_builder_matches_host(nb, which):
    if which == "edge":
        scene = _edge_scene(nb)
    elif which == "ico":
        scene = nb.synth_icospheres(seed=11, instances=64, extent=100.0)
    else:
        scene = nb.synth_city(seed=5, grid=8, size_m=250.0, target_tris=120_000, median_tris=1000,
                              max_tris=20_000, emissive_quads=8)
    _same(nb.SceneBVH(scene, device=0), nb.SceneBVH(scene))


def test_gpu_builder_bench_city(nb):
    """The 2.5M-triangle bench city: equal arrays, and the GPU build timed beside the host build."""
    scene = nb.synth_city(seed=2)
    nb.SceneBVH(nb.synth_icospheres(seed=1, instances=4), device=0)  # context and module load
    t0 = time.perf_counter()
    g = nb.SceneBVH(scene, device=0)
    t1 = time.perf_counter()
    h = nb.SceneBVH(scene)
    t2 = time.perf_counter()
    _same(g, h)
    print(f"scenebvh build: gpu {t1 - t0:.3f} s, host {t2 - t1:.3f} s")
