"""The bench's reference arm builds its workload without this repository's library: the seeded
city from the generator's source compiled on its own (oracle/_build/libsynth.so), the SceneBVH
arrays from the reference's own builder and the primary hits from the reference's own traversal.
Checked here: that workload equals the product arm's, and building it maps no product library."""
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CITY = dict(seed=5, grid=6, size_m=200.0, target_tris=40_000, median_tris=600, max_tris=8_000, emissive_quads=4)


def test_workload_scene_equals_product_scene(nb):
    from oracle import workload as wl

    a, b = wl.synth_city(**CITY), nb.synth_city(**CITY)
    for k in ("prim_type", "prim_geom", "prim_material", "object_first", "object_prims"):
        assert np.array_equal(np.asarray(getattr(a, k)).view(np.uint8), np.asarray(getattr(b, k)).view(np.uint8)), k


def test_workload_scenebvh_and_rays_equal_product(nb, orc):
    from oracle import reference as ref
    from oracle import workload as wl

    if not ref.available():
        pytest.skip("reference build (oracle/_ref) not present")
    sb_ref = wl.scene_bvh(wl.synth_city(**CITY))
    sb = nb.SceneBVH(nb.synth_city(**CITY))
    for k in ("bvh_nodes", "tlas_nodes", "prims", "materials", "prim_indices", "prim_object"):
        assert np.array_equal(np.asarray(getattr(sb_ref, k)).view(np.uint8), np.asarray(getattr(sb, k)).view(np.uint8)), k
    assert np.array_equal(sb_ref.instances["blas_root_index"], sb.instances["blas_root_index"])
    cam = nb.Camera((0, 50, -150), (0, 0, 0), width=64, height=40)
    rays = wl.city_rays(sb_ref, cam, 1, 3, 4)
    prim = cam.primary_rays(1, seed=3)
    want = np.concatenate([prim, nb.bounce_rays(prim, orc.OracleScene(sb).closest(prim), sb.prims, seed=4)])
    assert rays.shape == want.shape
    # the bounces follow the reference's hits; they differ from the contract's only on tied rays
    assert (rays.view(np.uint8).reshape(rays.shape[0], -1) == want.view(np.uint8).reshape(want.shape[0], -1)).all(1).mean() > 0.99


def test_reference_arm_maps_no_product_library():
    from oracle import reference as ref

    if not ref.available():
        pytest.skip("reference build (oracle/_ref) not present")
    code = (
        "import re, sys; sys.path.insert(0, %r)\n"
        "from oracle import workload as wl, reference as ref\n"
        "from nomad_b200.rays import Camera\n"
        "sb = wl.scene_bvh(wl.synth_city(**%r))\n"
        "rays = wl.city_rays(sb, Camera((0, 50, -150), (0, 0, 0), width=32, height=20), 1, 3, 4)\n"
        "ref.closest(sb, rays)\n"
        "print('\\n'.join(sorted(set(re.findall(r'(/\\S+\\.so)', open('/proc/self/maps').read())))))\n"
    ) % (ROOT, CITY)
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, check=True).stdout
    mine = [line for line in out.split() if line.startswith(ROOT)]
    assert mine and all(line.startswith(os.path.join(ROOT, "oracle")) for line in mine), mine


def test_cpu_baseline_extras(nb, orc):
    """The CPU baseline's any-hit rate and path-traced frame estimate run on a small city: the
    any-hit answers agree with the closest hits (a ray with a closest hit is occluded), and the
    frame estimate is the sampled pixels' time scaled to the full frame."""
    sys.path.insert(0, ROOT)
    import bench

    sb = nb.SceneBVH(nb.synth_city(**CITY))
    os_ = orc.OracleScene(sb)
    cam = nb.Camera((0, 50, -150), (0, 0, 0), width=64, height=40)
    rays = cam.primary_rays(1, seed=3)
    hit = os_.closest(rays)["prim"] >= 0
    assert np.array_equal(os_.any(rays).astype(bool), hit)
    out = bench.cpu_extra(os_, orc, sb, rays, 2, budget_s=0.2)
    assert out["any_hit_mrays_s"] > 0 and out["path_traced_ms_per_frame"] > 0
    assert "seeded pixels of the C2 frame" in out["path_traced_sample"]
