"""ORACLE recipe — test infrastructure only. Loads every scene XML shipped with the reference
(under $NOMAD_REFERENCE/Nomad Path Tracer, default /root/reference, where the reference tree is
present) with both the
reference's own loader (oracle/_ref/libref_ingest.so, built by `make -C oracle ref`) and
nomad_scene_load_xml, and compares the results array by array, bit for bit. Prints one line per
scene with the primitive and object counts, the two load times and the verdict.

    python oracle/ref/check_reference_scenes.py [scene.xml ...]
"""
import glob
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import nomad_b200 as nb  # noqa: E402
from oracle import reference_ingest as ri  # noqa: E402

REF_SCENES = os.path.join(os.environ.get("NOMAD_REFERENCE", "/root/reference"), "Nomad Path Tracer")
ARRAYS = ("prim_type", "prim_geom", "prim_material", "object_first", "object_prims", "object_mesh_group")


def quiet(fn, *a):
    """Runs fn with the process's stdout sent to /dev/null (the reference loader prints per mesh)."""
    sys.stdout.flush()
    saved = os.dup(1)
    null = os.open(os.devnull, os.O_WRONLY)
    os.dup2(null, 1)
    try:
        return fn(*a)
    finally:
        os.dup2(saved, 1)
        os.close(null)
        os.close(saved)


def compare(path):
    t0 = time.perf_counter()
    try:
        mine = nb.load_scene_xml(path)
    except nb.NomadError:
        mine = None
    t1 = time.perf_counter()
    ref = quiet(ri.load_xml, path)
    t2 = time.perf_counter()
    name = os.path.basename(path)
    if ref is None or mine is None:
        if ref is None and mine is None:
            return f"{name}: both loaders reject the file; agree"
        return f"{name}: DIFFERS: only {'the reference' if ref is None else 'nomad_scene_load_xml'} rejects it"
    bad = [k for k in ARRAYS
           if getattr(mine, k).shape[0] != ref[k].shape[0]
           or not np.array_equal(np.ascontiguousarray(getattr(mine, k)).view(np.uint8),
                                 np.ascontiguousarray(ref[k]).view(np.uint8))]
    for k in ("settings", "keyframes", "observer", "environment_texture"):
        if getattr(mine, k) != ref[k]:
            bad.append(k)
    verdict = "bit-exact" if not bad else "DIFFERS in " + ", ".join(bad)
    return (f"{name}: {mine.prim_count} primitives, {mine.object_count} objects, "
            f"{mine.mesh_files} OBJ files ({mine.mesh_files_failed} missing); "
            f"load {t1 - t0:.2f} s here vs {t2 - t1:.2f} s reference; {verdict}")


def main():
    paths = sys.argv[1:] or sorted(glob.glob(os.path.join(REF_SCENES, "*.xml")))
    for p in paths:
        print(compare(p), flush=True)


if __name__ == "__main__":
    main()
