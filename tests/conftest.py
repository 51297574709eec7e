import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def nb():
    import nomad_b200

    nomad_b200.load()
    return nomad_b200


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle

    oracle.load()
    return oracle


@pytest.fixture(scope="session")
def ico_scene(nb):
    scene = nb.synth_icospheres(seed=11, instances=64, extent=100.0)
    return scene, nb.SceneBVH(scene)


@pytest.fixture(scope="session")
def small_city(nb):
    scene = nb.synth_city(seed=5, grid=8, size_m=250.0, target_tris=120_000, median_tris=1000,
                          max_tris=20_000, emissive_quads=8)
    return scene, nb.SceneBVH(scene)
