"""CPU tests: the scene builder's invariants and the oracle's self-consistency.

The oracle restates the reference traversal in three orders (reference order, near-first,
brute force); the contract says the closest hit may not depend on the order, so all three must
agree bit for bit on every ray.
"""
import numpy as np
import pytest

from tests import raysets


def _bits(h):
    return np.ascontiguousarray(h).view(np.int32).reshape(-1, 5)


def _rays(sb, seed, n=4000):
    return np.concatenate([raysets.aimed_rays(sb, n, seed), raysets.random_rays(sb, n, seed + 1),
                           raysets.edge_case_rays(sb, seed + 2)])


def test_scenebvh_invariants(ico_scene, small_city):
    for scene, sb in (ico_scene, small_city):
        n = sb.prim_count
        assert np.array_equal(np.sort(sb.prim_indices), np.arange(n, dtype=np.int32))
        nodes = sb.bvh_nodes.reshape(-1, 8)
        a = nodes[:, 3].view(np.int32)
        b = nodes[:, 7].view(np.int32)
        leaf = b > 0
        # leaves tile every object's primitive range
        covered = np.zeros(n, np.int32)
        for f, c in zip(a[leaf], b[leaf]):
            covered[f:f + c] += 1
        assert (covered == 1).all()
        # every child box lies inside its parent box (the order-independence argument needs it)
        inner = np.nonzero(~leaf)[0]
        for ch in (a[inner], -b[inner]):
            assert (ch > inner).all()
            assert (nodes[ch, :3] >= nodes[inner, :3]).all()
            assert (nodes[ch, 4:7] <= nodes[inner, 4:7]).all()
        # TLAS leaves encode (-(obj+1), obj) and their boxes equal the BLAS root boxes
        t = sb.tlas_nodes.reshape(-1, 8)
        tl = t[:, 3].view(np.int32)
        tr = t[:, 7].view(np.int32)
        lf = tl < 0
        assert np.array_equal(-(tl[lf] + 1), tr[lf])
        assert sorted(tr[lf].tolist()) == list(range(sb.object_count))
        roots = sb.instances["blas_root_index"][tr[lf]]
        assert np.array_equal(t[lf][:, [0, 1, 2, 4, 5, 6]], nodes[roots][:, [0, 1, 2, 4, 5, 6]])
        # packed primitive type tags
        p = sb.prims.reshape(-1, 7, 4)
        assert set(np.unique(p[:, 0, 3]).tolist()) <= {0.0, 1.0, 2.0}


def test_builder_is_deterministic(nb):
    s1 = nb.SceneBVH(nb.synth_icospheres(3, 8, 20.0), threads=1)
    s2 = nb.SceneBVH(nb.synth_icospheres(3, 8, 20.0), threads=4)
    for k in ("bvh_nodes", "tlas_nodes", "prims", "materials", "prim_indices"):
        assert np.array_equal(getattr(s1, k).view(np.uint8), getattr(s2, k).view(np.uint8)), k


@pytest.mark.parametrize("which", ["ico", "city"])
def test_oracle_orders_agree(orc, ico_scene, small_city, which):
    scene, sb = ico_scene if which == "ico" else small_city
    rays = _rays(sb, 100)
    o = orc.OracleScene(sb)
    h0 = o.closest(rays, orc.MODE_REFERENCE_ORDER)
    h1 = o.closest(rays, orc.MODE_NEAR_FIRST)
    h2 = o.closest(rays, orc.MODE_BRUTE)
    assert (h0["prim"] >= 0).mean() > 0.2
    assert np.array_equal(_bits(h0), _bits(h1))
    assert np.array_equal(_bits(h0), _bits(h2))
    a0 = o.any(rays, orc.MODE_REFERENCE_ORDER)
    assert np.array_equal(a0, o.any(rays, orc.MODE_NEAR_FIRST))
    assert np.array_equal(a0, o.any(rays, orc.MODE_BRUTE))
    # with tmax = inf an any-hit exists exactly when a closest hit exists
    fin = np.isinf(rays["tmax"])
    assert np.array_equal(a0[fin].astype(bool), h0["prim"][fin] >= 0)


def test_oracle_residency(orc, small_city):
    scene, sb = small_city
    rays = _rays(sb, 7, n=3000)
    rng = np.random.default_rng(3)
    active = np.ones(sb.prim_count, np.uint8)
    active[rng.random(sb.prim_count) < 0.2] = 0
    root = sb.instances["blas_root_index"].copy()
    root[rng.random(sb.object_count) < 0.3] = -1
    o = orc.OracleScene(sb, active=active, blas_root=root)
    h0 = o.closest(rays, orc.MODE_REFERENCE_ORDER)
    assert np.array_equal(_bits(h0), _bits(o.closest(rays, orc.MODE_BRUTE)))
    hit = h0["prim"] >= 0
    assert active[h0["prim"][hit]].all()
    assert (root[h0["inst"][hit]] >= 0).all()


def test_oracle_tie_rule(orc, nb):
    """Two coplanar triangles sharing an edge: a ray through the edge hits both at the same t;
    the lower primitive index wins."""
    geom = np.zeros((2, 15), np.float32)
    geom[0, :9] = [0, 0, 0, 1, 0, 0, 0, 1, 0]
    geom[1, :9] = [1, 0, 0, 1, 1, 0, 0, 1, 0]
    mat = np.zeros((2, 20), np.float32)
    mat[:, 16:19] = -1
    for order in ([0, 1], [1, 0]):
        scene = nb.HostScene(np.ones(2, np.int32), geom[order], mat, [0], [2])
        sb = nb.SceneBVH(scene)
        rays = raysets._pack([[0.5, 0.5, 1.0], [0.25, 0.25, 1.0]], [[0, 0, -1], [0, 0, -1]])
        h = orc.OracleScene(sb).closest(rays)
        assert h["prim"][0] == 0 and h["t"][0] == np.float32(1.0)
        assert h["prim"][1] == order.index(0)


def test_work_counters_match_hits(orc, small_city):
    scene, sb = small_city
    rays = _rays(sb, 21, n=2000)
    o = orc.OracleScene(sb)
    w, h = o.work(rays)
    assert np.array_equal(_bits(h), _bits(o.closest(rays)))
    assert np.array_equal(w[:, 3].astype(bool), h["prim"] >= 0)
    assert (w[:, 0] >= 1).all() or (rays["tmax"] <= 1e-4).any()
