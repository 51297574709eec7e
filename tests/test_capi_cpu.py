"""CPU tests of the C ABI: the library loads, exports every declared symbol, and fails loudly
(never falls back) when no GPU is present."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    names = set()
    for h in ("nomad_rt.h", "nomad_scene.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(nomad_[a-z0-9_]+)\s*\(", src))
    return names


def test_exports_every_declared_symbol(nb):
    lib = ctypes.CDLL(nb.LIB_PATH)
    declared = _declared_symbols()
    assert len(declared) >= 24
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing
    assert declared == set(nb.SIGNATURES), declared ^ set(nb.SIGNATURES)


def test_no_gpu_fails_loudly(nb):
    import torch

    if torch.cuda.is_available():
        pytest.skip("GPU present")
    with pytest.raises(nb.NomadError):
        nb.Context(0)


def test_scene_validation(nb):
    geom = np.zeros((2, 15), np.float32)
    geom[:, :9] = [0, 0, 0, 1, 0, 0, 0, 1, 0]
    mat = np.zeros((2, 20), np.float32)
    bad_type = nb.HostScene(np.array([1, 7], np.int32), geom, mat, [0], [2])
    with pytest.raises(nb.NomadError):
        nb.SceneBVH(bad_type)
    gap = nb.HostScene(np.ones(2, np.int32), geom, mat, [0, 1], [1, 2])
    with pytest.raises(nb.NomadError):
        nb.SceneBVH(gap)
    nan = geom.copy()
    nan[0, 0] = np.nan
    with pytest.raises(nb.NomadError):
        nb.SceneBVH(nb.HostScene(np.ones(2, np.int32), nan, mat, [0], [2]))


def test_synthetic_scene_sizes(nb):
    s = nb.synth_icospheres(1, 64, 100.0)
    assert s.prim_count == 64 * 1280 and s.object_count == 64
    c = nb.synth_city(2)
    assert c.object_count == 1024
    assert 2_300_000 < c.prim_count < 2_700_000
    assert (c.prim_type == 2).sum() == 64
    mats = c.prim_material
    assert ((mats[:, 11] > 0) & (c.prim_type == 2)).sum() == 64
