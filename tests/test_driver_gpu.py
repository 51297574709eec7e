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
