"""Writes the golden results of the ingest fixtures in this folder: each scene XML loaded by the
reference's own loader (SceneLoader::LoadSceneFromXML with the vendored tinyxml2 and
tinyobjloader, compiled here by `make -C oracle ref`). The tests compare nomad_scene_load_xml
against these files bit for bit.

    python tests/golden/ingest/make_golden.py

Writes <name>.npz (arrays) and <name>.json (settings, camera path, observer, environment texture
relative to this folder) for every fixture the reference accepts, and records the rejected ones
in rejected.json.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, ROOT)

from oracle import reference_ingest as ri  # noqa: E402

FIXTURES = ("edge.xml", "defaults.xml", "broken.xml", "noscene.xml")
ARRAYS = ("prim_type", "prim_geom", "prim_material", "object_first", "object_prims", "object_mesh_group")


def main():
    rejected = []
    for name in FIXTURES:
        path = os.path.join(HERE, name)
        ref = ri.load_xml(path)
        stem = os.path.splitext(name)[0]
        if ref is None:
            rejected.append(name)
            continue
        np.savez(os.path.join(HERE, stem + ".npz"), **{k: ref[k] for k in ARRAYS})
        env = ref["environment_texture"]
        meta = {"settings": ref["settings"], "keyframes": ref["keyframes"], "observer": ref["observer"],
                "environment_texture": os.path.relpath(env, HERE) if env else ""}
        with open(os.path.join(HERE, stem + ".json"), "w") as f:
            json.dump(meta, f, indent=1, sort_keys=True)
        print(f"{name}: {ref['prim_type'].shape[0]} primitives, {ref['object_first'].shape[0]} objects")
    with open(os.path.join(HERE, "rejected.json"), "w") as f:
        json.dump(rejected, f)
    print("rejected:", rejected)


if __name__ == "__main__":
    main()
