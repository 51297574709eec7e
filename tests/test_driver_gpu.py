"""The C++ frame-loop driver (nomad_b200/bin/nomad_frame_loop): a host program that renders and
runs residency steps through the C ABI only. Its last frame must equal the same view rendered
through the Python binding, bit for bit."""
import json
import os
import subprocess
import tempfile

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "nomad_b200", "bin",
                      "nomad_frame_loop")


def _run(*args):
    assert os.path.exists(DRIVER), "build the driver with make -C nomad_b200/csrc"
    out = subprocess.run([DRIVER, *args], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    return json.loads(out.stdout.strip().splitlines()[-1])


def _read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline().strip() == b"PF"
        w, h = (int(x) for x in f.readline().split())
        scale = float(f.readline())
        assert scale < 0  # little-endian
        data = np.frombuffer(f.read(), "<f4").reshape(h, w, 3)
    return data[::-1]  # stored bottom row first


def test_driver_matches_binding(nb):
    with tempfile.TemporaryDirectory() as d:
        pfm = os.path.join(d, "last.pfm")
        r = _run("--scene", "icospheres", "--width", "96", "--height", "54", "--spp", "2", "--depth", "3",
                 "--frames", "3", "--policy", "always", "--seed", "17", "--out", pfm)
        img = _read_pfm(pfm)
    assert r["status"] == 0 and r["resident_fraction"] == 1.0
    scene = nb.synth_icospheres(seed=17, instances=64, extent=100.0)
    sb = nb.SceneBVH(scene)
    ctx = nb.Context(0)
    try:
        ctx.upload(sb)
        v = nb.view_pinhole((0, 0, 10), (0, 0, 0), width=96, height=54)
        for key in ("camera_pos", "viewport_u", "viewport_v", "first_pixel"):
            v[key] = np.asarray(r["view"][key], np.float32)
        v["spp"], v["max_depth"], v["seed_lo"], v["frame"] = 2, 3, 17, r["last_frame"]
        want = ctx.render(v)[0]
    finally:
        ctx.close()
    assert np.array_equal(img.view(np.int32), want.view(np.int32))
    assert abs(float(want.astype(np.float64).sum()) - r["radiance_sum"]) <= 1e-4 * max(1.0, r["radiance_sum"])


def test_driver_budget_policy():
    r = _run("--scene", "city", "--width", "160", "--height", "90", "--spp", "1", "--depth", "2", "--frames", "6",
             "--policy", "rayhit", "--budget", "0.4")
    assert r["status"] == 0
    assert 0.0 < r["resident_fraction"] <= 0.4 + 1e-9
    assert r["render_ms_per_frame"] > 0 and r["rays"] > 0


def test_driver_renders_an_ingested_scene_like_the_binding(nb):
    """--scene xml:FILE: the scene file's camera path and size drive the loop; the last frame equals
    the binding's render of the same loaded scene and view."""
    xml = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ingest", "edge.xml")
    with tempfile.TemporaryDirectory() as d:
        pfm = os.path.join(d, "last.pfm")
        r = _run("--scene", "xml:" + xml, "--spp", "1", "--frames", "20", "--policy", "always", "--seed", "5",
                 "--out", pfm)
        img = _read_pfm(pfm)
    s = nb.load_scene_xml(xml)
    assert r["status"] == 0 and r["prims"] == s.prim_count and r["objects"] == s.object_count
    assert (r["width"], r["height"], r["depth"]) == (640, 360, 6)
    sb = nb.SceneBVH(s)
    ctx = nb.Context(0)
    try:
        ctx.upload(sb)
        v = nb.view_pinhole((0, 0, 10), (0, 0, 0), width=640, height=360)
        for key in ("camera_pos", "viewport_u", "viewport_v", "first_pixel"):
            v[key] = np.asarray(r["view"][key], np.float32)
        v["spp"], v["max_depth"], v["seed_lo"], v["frame"] = 1, 6, 5, r["last_frame"]
        want = ctx.render(v)[0]
    finally:
        ctx.close()
    assert np.array_equal(img.view(np.int32), want.view(np.int32))


def test_driver_learned_policy_from_a_model_file(nb, tmp_path):
    """--mlp takes a model file written by nomad_mlp_save."""
    ctx = nb.Context(0)
    try:
        ctx.mlp_init(7)
        path = str(tmp_path / "scorer.nmlp")
        ctx.mlp_save(path)
    finally:
        ctx.close()
    r = _run("--scene", "city", "--width", "160", "--height", "90", "--spp", "1", "--depth", "2", "--frames", "4",
             "--policy", "learned", "--budget", "0.4", "--mlp", path)
    assert r["status"] == 0 and 0.0 < r["resident_fraction"] <= 0.4 + 1e-9
