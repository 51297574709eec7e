"""Scene ingest (nomad_scene_load_xml): XML scenes with OBJ/MTL meshes.

CPU: the loader against golden results that the reference's own loader (SceneLoader with the
vendored tinyxml2 and tinyobjloader, compiled here) produced from the fixtures in
tests/golden/ingest: every primitive's type, geometry and material, every object's range and mesh
group, the settings, camera path, observer camera and environment texture, bit for bit. The
fixtures cover quads and larger polygons (convex, concave, collinear, degenerate, with an
out-of-range index), the index forms and negative indices, CRLF endings, vertex colours, the
number formats of tinyobjloader's parser, material libraries (missing files, duplicate names,
`d` against `Tr`, `map_Kd` without `Kd`, unknown and empty `usemtl` names, fallbacks), faces that
reference vertices defined later, a file that fails to parse, a missing file, mesh baking by
scale, rotation and basis vectors, object splitting by triangle count and extent, and
hexadecimal, boolean, entity-encoded and malformed attributes. Rejected documents (mismatched
tags, no <Scene> root) are rejected by both loaders.
GPU: a loaded fixture scene traced on the device equals the oracle's traversal.
"""
import json
import os

import numpy as np
import pytest

from tests import raysets

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ingest")
ARRAYS = ("prim_type", "prim_geom", "prim_material", "object_first", "object_prims", "object_mesh_group")


def _same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _check_against(s, arrays, meta):
    for k in ARRAYS:
        got = getattr(s, k)
        want = arrays[k]
        assert _same_bits(got.reshape(want.shape) if got.size == want.size else got, want), k
    assert s.settings == meta["settings"]
    assert [dict(k, position=list(k["position"]), look_at=list(k["look_at"]), up=list(k["up"]))
            for k in s.keyframes] == meta["keyframes"]
    obs = s.observer
    if obs is not None:
        obs = dict(obs, position=list(obs["position"]), look_at=list(obs["look_at"]), up=list(obs["up"]))
    assert obs == meta["observer"]
    env = os.path.relpath(s.environment_texture, GOLDEN) if s.environment_texture else ""
    assert env == meta["environment_texture"]


@pytest.mark.parametrize("name", ["edge", "defaults"])
def test_matches_reference_loader_golden(nb, name):
    s = nb.load_scene_xml(os.path.join(GOLDEN, name + ".xml"))
    arrays = np.load(os.path.join(GOLDEN, name + ".npz"))
    with open(os.path.join(GOLDEN, name + ".json")) as f:
        meta = json.load(f)
    _check_against(s, arrays, meta)


def test_edge_fixture_exercises_the_reader(nb):
    """The edge fixture reaches the paths it is meant to cover."""
    s = nb.load_scene_xml(os.path.join(GOLDEN, "edge.xml"))
    assert s.mesh_files == 6 and s.mesh_files_failed == 2  # bad_index.obj fails, not_there.obj is missing
    assert "out-of-range vertex indices dropped" in s.log
    groups = s.object_mesh_group
    assert (groups == -1).sum() == 5                       # 3 spheres + 2 rectangles, one object each
    counts = np.bincount(groups[groups >= 0])
    assert counts.max() > 1                                # a mesh split into several objects
    assert s.settings["residency_strategy"] == 3 and s.settings["max_ray_depth"] == 6
    assert s.settings["environment_brightness"] == 0.0 and s.settings["start_compacted"] == 1
    assert s.environment_texture.endswith("sky&sun.exr")
    assert len(s.keyframes) == 3 and s.keyframes[2]["frame"] == 64


def test_defaults_of_an_empty_scene(nb):
    s = nb.load_scene_xml(os.path.join(GOLDEN, "defaults.xml"))
    assert s.prim_count == 0 and s.object_count == 0 and s.observer is None
    st = s.settings
    assert (st["width"], st["height"], st["max_ray_depth"], st["residency_strategy"]) == (1280.0, 720.0, 32, 0)
    assert st["max_tile_work"] == 64 * 64 * 4 and st["total_gpu_cap_mb"] == 4096.0


def test_rejected_documents(nb):
    with open(os.path.join(GOLDEN, "rejected.json")) as f:
        rejected = json.load(f)
    assert sorted(rejected) == ["broken.xml", "noscene.xml"]
    why = {"broken.xml": "mismatched end tag", "noscene.xml": "no <Scene> root", "does_not_exist.xml": "cannot read"}
    for name in rejected + ["does_not_exist.xml"]:
        with pytest.raises(nb.NomadError, match=why[name]):
            nb.load_scene_xml(os.path.join(GOLDEN, name))


def test_deep_nesting_is_rejected_not_crashed(nb, tmp_path):
    """Nesting deeper than 500 elements is refused with a message (the reader is recursive)."""
    deep = tmp_path / "deep.xml"
    deep.write_text("<Scene>" + "<a>" * 20000 + "</a>" * 20000 + "</Scene>")
    with pytest.raises(nb.NomadError, match="nested too deeply"):
        nb.load_scene_xml(str(deep))
    ok = tmp_path / "ok.xml"
    ok.write_text("<Scene>" + "<a>" * 400 + "</a>" * 400 + '<Sphere position="0,0,0"/></Scene>')
    assert nb.load_scene_xml(str(ok)).prim_count == 1


def test_thread_count_does_not_change_the_result(nb):
    path = os.path.join(GOLDEN, "edge.xml")
    a, b = nb.load_scene_xml(path, threads=1), nb.load_scene_xml(path, threads=7)
    for k in ARRAYS:
        assert _same_bits(getattr(a, k), getattr(b, k)), k


def test_loaded_scene_builds_a_scenebvh(nb):
    s = nb.load_scene_xml(os.path.join(GOLDEN, "edge.xml"))
    sb = nb.SceneBVH(s)
    assert sb.prim_count == s.prim_count and sb.object_count == s.object_count


def test_reference_loader_live(nb):
    """Where the reference's loader was compiled here, run it on the fixtures directly."""
    from oracle import reference_ingest as ri

    if not ri.available():
        pytest.skip("oracle/_ref/libref_ingest.so not built")
    for name in ("edge", "defaults"):
        path = os.path.join(GOLDEN, name + ".xml")
        ref = ri.load_xml(path)
        s = nb.load_scene_xml(path)
        for k in ARRAYS:
            assert _same_bits(getattr(s, k).reshape(ref[k].shape), ref[k]), (name, k)
        assert s.settings == ref["settings"]


@pytest.mark.gpu
def test_ingested_scene_traces_like_the_oracle(nb, orc):
    s = nb.load_scene_xml(os.path.join(GOLDEN, "edge.xml"))
    sb = nb.SceneBVH(s)
    rays = np.concatenate([raysets.aimed_rays(sb, 20000, 71), raysets.random_rays(sb, 20000, 72)])
    ctx = nb.Context(0)
    try:
        ctx.upload(sb)
        got = ctx.trace_closest(rays)
        occl = ctx.trace_any(rays)
    finally:
        ctx.close()
    ref = orc.OracleScene(sb)
    want = ref.closest(rays)
    assert np.array_equal(np.ascontiguousarray(got).view(np.int32), np.ascontiguousarray(want).view(np.int32))
    assert np.array_equal(occl, ref.any(rays))
    assert (want["inst"] >= 0).mean() > 0.3
