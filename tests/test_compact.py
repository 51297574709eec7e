"""Residency compaction: the oracle's restatement of the reference's compacted path and the
device compaction (nomad_scenebvh_compact_gpu) against it.

CPU: tracing the compacted arrays (every primitive active) must give the same closest hits as
tracing the full arrays under the active mask, once compact primitive indices are mapped back
through the remap; plus the structural properties of the compacted arrays.
GPU: the device compaction equals the oracle's, bit for bit, on per-primitive and per-object
masks, the empty and the full mask, and the 2.5M-triangle city; and the compacted scene traced
on the device gives the masked full scene's hits.
"""
import types

import numpy as np
import pytest

from tests import raysets


def _masks(sb, seed):
    rng = np.random.default_rng(seed)
    n, nobj = sb.prim_count, sb.object_count
    per_prim = (rng.random(n) < 0.5).astype(np.uint8)
    objs = rng.random(nobj) < 0.4
    per_obj = objs[sb.prim_object].astype(np.uint8)
    # objects mostly off, a few primitives on inside some of them
    sparse = (rng.random(n) < 0.03).astype(np.uint8)
    return {"per_prim": per_prim, "per_object": per_obj, "sparse": sparse,
            "all": np.ones(n, np.uint8), "none": np.zeros(n, np.uint8)}


def _compact_scene(sb, c):
    """A SceneBVH-like view of compacted arrays (TLAS unchanged) for the oracle traversal."""
    prim_object = sb.prim_object[c["remap"].astype(np.int64)] if c["prim_count"] else np.zeros(0, np.int32)
    return types.SimpleNamespace(
        bvh_nodes=c["bvh_nodes"] if c["bvh_node_count"] else np.zeros(8, np.float32),
        tlas_nodes=sb.tlas_nodes, prims=c["prims"] if c["prim_count"] else np.zeros(28, np.float32),
        prim_indices=c["prim_indices"] if c["prim_count"] else np.zeros(1, np.int32),
        prim_object=np.ascontiguousarray(prim_object, np.int32) if c["prim_count"] else np.zeros(1, np.int32),
        object_count=sb.object_count, prim_count=max(c["prim_count"], 1), instances=c["instances"])


def _check_structure(sb, active, c):
    n = sb.prim_count
    act = active.astype(bool)
    p = c["prim_count"]
    assert p == int(act.sum())
    # remap lists the active primitives in object order, BLAS-leaf order inside an object
    leaf_order = sb.prim_indices[act[sb.prim_indices]]
    assert np.array_equal(c["remap"], leaf_order.astype(np.uint32))
    assert np.array_equal(c["prim_indices"], np.arange(p, dtype=np.int32))
    p2r = np.full(n, -1, np.int32)
    p2r[c["remap"].astype(np.int64)] = np.arange(p, dtype=np.int32)
    assert np.array_equal(c["prim_to_resident"], p2r)
    g = c["remap"].astype(np.int64)
    assert np.array_equal(c["prims"].reshape(p, 28), sb.prims.reshape(n, 28)[g])
    assert np.array_equal(c["materials"].reshape(p, 20), sb.materials.reshape(n, 20)[g])
    inst = c["instances"]
    per_obj = np.bincount(sb.prim_object[act], minlength=sb.object_count)
    assert np.array_equal(inst["primitive_count"], per_obj.astype(np.uint32))
    assert np.array_equal(inst["primitive_base"], inst["primitive_index_base"])
    assert ((inst["blas_root_index"] >= 0) == (per_obj > 0)).all()
    # children precede their parents (post-order); leaves tile the compact primitive range
    nodes = c["bvh_nodes"].reshape(-1, 8)
    a = nodes[:, 3].view(np.int32)
    b = nodes[:, 7].view(np.int32)
    leaf = b > 0
    idx = np.arange(nodes.shape[0])
    assert (a[~leaf] < idx[~leaf]).all() and (-b[~leaf] < idx[~leaf]).all()
    covered = np.zeros(p, np.int32)
    for f, k in zip(a[leaf], b[leaf]):
        covered[f:f + k] += 1
    assert (covered == 1).all()


def _same_hits(full, comp, remap):
    """Closest hits equal up to exact-t ties. Ties go to the lowest primitive index, and the
    compact order (object, then BLAS leaf order) is not the global order, so on a tie the full
    scene keeps the lowest global index and the compacted one the lowest compact index."""
    assert np.array_equal(full["t"].view(np.int32), comp["t"].view(np.int32))
    hit = comp["inst"] >= 0
    assert np.array_equal(full["inst"] >= 0, hit)
    g = np.full(comp.shape[0], -1, np.int64)
    g[hit] = remap[comp["prim"][hit]].astype(np.int64)
    same = (g == full["prim"]) & (comp["inst"] == full["inst"])
    inv = np.full(int(remap.max()) + 1 if remap.size else 1, -1, np.int64)
    inv[remap.astype(np.int64)] = np.arange(remap.size)
    tie = ~same
    assert (g[tie] > full["prim"][tie]).all()                    # full kept the lower global id
    assert (inv[full["prim"][tie]] > comp["prim"][tie]).all()    # compact kept the lower compact id
    assert tie.sum() <= max(4, comp.shape[0] // 200)
    both = same & hit
    for k in ("u", "v"):
        assert np.array_equal(full[k][both].view(np.int32), comp[k][both].view(np.int32))


@pytest.mark.parametrize("scene", ["ico", "city"])
def test_oracle_compaction_traces_like_the_mask(orc, ico_scene, small_city, scene):
    _, sb = ico_scene if scene == "ico" else small_city
    rays = np.concatenate([raysets.aimed_rays(sb, 3000, 31), raysets.random_rays(sb, 3000, 32)])
    for name, active in _masks(sb, 7).items():
        c = orc.compact(sb, active)
        _check_structure(sb, active, c)
        full = orc.OracleScene(sb, active=active).closest(rays)
        if c["prim_count"] == 0:
            assert (full["inst"] < 0).all(), name
            continue
        cs = _compact_scene(sb, c)
        comp = orc.OracleScene(cs, blas_root=c["instances"]["blas_root_index"]).closest(rays)
        _same_hits(full, comp, c["remap"])


def test_oracle_compaction_all_active_keeps_the_tree(orc, ico_scene):
    """With every primitive active nothing is pruned: the same nodes, renumbered in post-order."""
    _, sb = ico_scene
    c = orc.compact(sb, np.ones(sb.prim_count, np.uint8))
    assert c["bvh_node_count"] == sb.bvh_node_count
    full = sb.bvh_nodes.reshape(-1, 8)
    comp = c["bvh_nodes"].reshape(-1, 8)
    key = lambda m: np.unique(m[:, [0, 1, 2, 4, 5, 6]].view(np.int32), axis=0)
    assert np.array_equal(key(full), key(comp))
    # each object's root is its last node
    roots = c["instances"]["blas_root_index"]
    ends = np.cumsum(np.diff(np.append(np.sort(sb.instances["blas_root_index"]), sb.bvh_node_count)))
    assert np.array_equal(np.sort(roots) + 1, ends)


# ---------------------------------------------------------------------------------------------
# GPU


def _device_vs_oracle(nb, orc, sb, masks):
    comp = nb.native.Compactor(sb)
    for name, active in masks.items():
        comp.run(active)
        got = comp.result()
        want = orc.compact(sb, active)
        assert got["prim_count"] == want["prim_count"], name
        assert got["bvh_node_count"] == want["bvh_node_count"], name
        for k in ("bvh_nodes", "prims", "materials", "prim_indices", "remap", "prim_to_resident"):
            assert np.array_equal(np.ascontiguousarray(got[k]).view(np.uint8),
                                  np.ascontiguousarray(want[k]).view(np.uint8)), (name, k)
        assert np.array_equal(got["instances"].view(np.int32), want["instances"].view(np.int32)), name
    return comp


@pytest.mark.gpu
@pytest.mark.parametrize("scene", ["ico", "city"])
def test_device_compaction_matches_oracle(nb, orc, ico_scene, small_city, scene):
    _, sb = ico_scene if scene == "ico" else small_city
    _device_vs_oracle(nb, orc, sb, _masks(sb, 19))


@pytest.mark.gpu
def test_device_compaction_full_city(nb, orc):
    """The 2.5M-triangle city under a 40 % object mask and a 50 % primitive mask."""
    sb = nb.SceneBVH(nb.synth_city(seed=7))
    rng = np.random.default_rng(3)
    masks = {"objects40": (rng.random(sb.object_count) < 0.4)[sb.prim_object].astype(np.uint8),
             "prims50": (rng.random(sb.prim_count) < 0.5).astype(np.uint8)}
    _device_vs_oracle(nb, orc, sb, masks)


@pytest.mark.gpu
def test_compacted_scene_traces_like_the_mask_on_device(nb, orc, small_city):
    """Upload the device-compacted arrays as a scene and trace them on the device: the hits are
    the masked full scene's (device) hits after the remap."""
    _, sb = small_city
    rng = np.random.default_rng(5)
    active = (rng.random(sb.object_count) < 0.4)[sb.prim_object].astype(np.uint8)
    active &= (rng.random(sb.prim_count) < 0.8).astype(np.uint8)
    comp = nb.native.Compactor(sb)
    comp.run(active)
    c = comp.result()
    rays = np.concatenate([raysets.aimed_rays(sb, 20000, 41), raysets.random_rays(sb, 20000, 42)])
    ctx = nb.Context()
    try:
        ctx.upload(sb)
        for o in np.nonzero(np.bincount(sb.prim_object[active.astype(bool)], minlength=sb.object_count) == 0)[0]:
            ctx.set_object_active(int(o), False)
        obj_on = np.bincount(sb.prim_object[active.astype(bool)], minlength=sb.object_count) > 0
        for p in np.nonzero((active == 0) & obj_on[sb.prim_object])[0]:
            ctx.set_primitive_active(int(p), False)
        ctx.flush()
        full = ctx.trace_closest(rays)
    finally:
        ctx.close()
    cs = _compact_scene(sb, c)
    cs.materials = c["materials"]
    cs.bvh_node_count = c["bvh_node_count"]
    cs.tlas_node_count = sb.tlas_node_count
    cs.prim_count = c["prim_count"]
    ctx = nb.Context()
    try:
        ctx.upload(cs)
        got = ctx.trace_closest(rays)
    finally:
        ctx.close()
    _same_hits(full, got, c["remap"])


@pytest.mark.gpu
def test_device_compaction_reports_bad_arrays(nb, ico_scene):
    """Out-of-range primitive indices and instance ranges are reported in counts[2], not faulted
    on (the kernels range-check every index they follow)."""
    _, sb = ico_scene
    bad = types.SimpleNamespace(**{k: getattr(sb, k) for k in (
        "prim_count", "bvh_node_count", "object_count", "bvh_nodes", "prims", "materials", "prim_object")})
    bad.prim_indices = sb.prim_indices.copy()
    bad.prim_indices[5] = sb.prim_count + 5
    bad.instances = sb.instances
    comp = nb.native.Compactor(bad)
    comp.run(np.ones(sb.prim_count, np.uint8))
    with pytest.raises(nb.NomadError, match="error bits 1"):
        comp.result()
    bad.prim_indices = sb.prim_indices
    bad.instances = sb.instances.copy()
    bad.instances["primitive_count"][-1] += 1000
    comp = nb.native.Compactor(bad)
    comp.run(np.ones(sb.prim_count, np.uint8))
    with pytest.raises(nb.NomadError, match="error bits"):
        comp.result()
