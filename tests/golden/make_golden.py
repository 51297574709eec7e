"""Generates the golden fixtures in this folder from the reference's own code.

Run where the reference sources are present (it needs oracle/_ref/libref_nomad.so, built by
`make -C oracle ref` from SceneBVH.cpp, Scene.cpp and Shaders/PathTracing.h):

    python tests/golden/make_golden.py

For two seeded scenes it stores
  * sha256 of every SceneBVH array the reference's builder produced;
  * the reference traversal's closest hits (firstHitTLAS, verbatim) on a seeded ray set;
  * the contract oracle's closest hits on the same rays.
Rays are regenerated from their seeds by tests/raysets.py, so only hits are stored.

shading_ref.npz (needs oracle/_ref/libref_shade.so, from PathTraceKernel.metal, PathTracing.h and
Scatter.h): the reference's shading functions on the seeded cases of tests/shading_pin.py (digests
of the bit-exact ones, the first 2,000 cases of the others), its path-traced frames and its
ReSTIR reference-mode sequence (radiance, selected light and sample count per pixel, a digest of
the surface records), all on the seeded random-number tapes.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import nomad_b200 as nb  # noqa: E402
from oracle import oracle as orc, reference as ref  # noqa: E402
from oracle import reference_shade as rshade  # noqa: E402
from tests import raysets, shading_pin as sp  # noqa: E402

SCENES = {
    "ico": lambda: nb.synth_icospheres(seed=11, instances=64, extent=100.0),
    "city": lambda: nb.synth_city(seed=5, grid=8, size_m=250.0, target_tris=120_000,
                                  median_tris=1000, max_tris=20_000, emissive_quads=8),
}


def golden_rays(sb, seed):
    return np.concatenate([raysets.aimed_rays(sb, 3000, seed), raysets.random_rays(sb, 1000, seed + 1),
                           raysets.edge_case_rays(sb, seed + 2)])


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def main():
    manifest = {}
    for name, make in SCENES.items():
        scene = make()
        r = ref.build_scene(scene)
        manifest[name] = {k: sha(r[k]) for k in ("bvh_nodes", "tlas_nodes", "prims", "materials",
                                                    "prim_indices", "blas_root")}
        sb = nb.SceneBVH(scene)
        rays = golden_rays(sb, 1000)
        h_ref = ref.closest(sb, rays)
        h_con = orc.OracleScene(sb).closest(rays)
        np.savez_compressed(os.path.join(HERE, f"hits_{name}.npz"), ref=h_ref.view(np.int32),
                            contract=h_con.view(np.int32), ray_sha=np.array(sha(rays)))
    with open(os.path.join(HERE, "scenebvh_sha256.json"), "w") as f:
        json.dump(manifest, f, indent=1, sort_keys=True)
    d = sp.function_inputs()
    full = sp.reference_function_outputs(rshade, d)
    a = np.array(full["resv"], np.float32)  # slot 7 as 1 / area where valid (the oracle's form)
    valid = a[:, 15] > 0
    a[:, 7] = np.where(valid, np.float32(1) / np.where(valid, a[:, 7], np.float32(1)), np.float32(0))
    full["resv"] = a
    g = sp.golden_function_outputs(full)
    g.update(sp.golden_frames(sp.reference_frames(nb, orc, rshade)))
    np.savez_compressed(os.path.join(HERE, sp.GOLDEN_FILE), **g)


if __name__ == "__main__":
    main()
