"""Seeded random scenes through both scene loaders: nomad_scene_load_xml against the reference's
own loader (SceneLoader with the vendored tinyobjloader and tinyxml2, compiled here into
oracle/_ref/libref_ingest.so), bit for bit. Skipped where that library was not built.

Each scene is a handful of OBJ files with random decimal spellings (signs, leading and trailing
dots, exponents, more fraction digits than tinyobjloader's lookup table), random polygons
(triangles, quads, convex and concave n-gons, stars, collinear and repeated points, faces that
name vertices defined later), every index form including relative indices, material switches
over a random MTL library, and <Mesh> elements with random placement, scale, rotation, basis
vectors, overrides and object splitting; plus random spheres and rectangles.
"""
import math
import os

import numpy as np
import pytest

ARRAYS = ("prim_type", "prim_geom", "prim_material", "object_first", "object_prims", "object_mesh_group")


def _num(rng, x):
    """One of several spellings of x that tinyobjloader's parser accepts."""
    k = rng.integers(0, 8)
    if k == 0:
        return f"{x:.9g}"
    if k == 1:
        return f"{x:e}"
    if k == 2:
        return f"{x:.3f}"
    if k == 3:
        return f"{x:+.6f}"
    if k == 4:
        s = f"{abs(x):.12f}"
        s = s[1:] if s.startswith("0.") else s  # leading dot
        return ("-" if x < 0 else "") + s
    if k == 5:
        return f"{x:.20f}"  # beyond the parser's 8-entry table of tenths
    if k == 6:
        return f"{x * 1e3:.5f}E-03"
    return f"{x:.4E}"


def _polygon(rng, n):
    """n points on a random plane: convex, star (concave) or with repeated / collinear points."""
    kind = rng.integers(0, 4)
    ang = np.sort(rng.uniform(0, 2 * math.pi, n))
    r = np.ones(n)
    if kind == 1:
        r[::2] = 0.35  # star
    elif kind == 2:
        r = rng.uniform(0.2, 1.0, n)
    pts = np.stack([r * np.cos(ang), r * np.sin(ang), np.zeros(n)], 1)
    if kind == 3 and n > 4:
        pts[2] = pts[1]  # repeated point
        pts[4] = (pts[3] + pts[5 % n]) / 2  # collinear
    a, b = rng.normal(size=3), rng.normal(size=3)
    a /= np.linalg.norm(a)
    b -= a * (a @ b)
    b /= np.linalg.norm(b)
    return pts[:, :1] * a + pts[:, 1:2] * b + rng.normal(size=3)


def _write_obj(rng, path, mtl_names):
    lines = ["# random fuzz mesh"]
    if mtl_names:
        lines.append("mtllib lib.mtl")
    nv = nvt = nvn = 0
    pending = []
    for _ in range(rng.integers(5, 25)):
        if mtl_names and rng.random() < 0.3:
            lines.append("usemtl " + (mtl_names[rng.integers(0, len(mtl_names))] if rng.random() < 0.9 else "nosuch"))
        if rng.random() < 0.1:
            lines.append(rng.choice(["g grp", "o obj", "s 1", "s off"]))
        n = int(rng.choice([3, 3, 4, 4, 5, 6, 7, 8]))
        pts = _polygon(rng, n)
        base = nv
        for p in pts:
            lines.append("v " + " ".join(_num(rng, float(c)) for c in p))
            nv += 1
        for _ in range(n):
            lines.append(f"vt {_num(rng, float(rng.random()))} {_num(rng, float(rng.random()))}")
            nvt += 1
        lines.append("vn 0 0 1")
        nvn += 1
        form = rng.integers(0, 5)
        idx = []
        for j in range(n):
            v, t = base + j + 1, nvt - n + j + 1
            if form == 4:  # relative indices
                v, t = v - nv - 1, t - nvt - 1
            idx.append([f"{v}", f"{v}/{t}", f"{v}//{nvn}", f"{v}/{t}/{nvn}", f"{v}/{t}"][form])
        face = "f " + " ".join(idx)
        if rng.random() < 0.1:
            pending.append(face)  # emitted after more vertices exist
        else:
            lines.append(face)
    lines.extend(pending)
    with open(path, "w", newline="\r\n" if rng.random() < 0.3 else "\n") as f:
        f.write("\n".join(lines) + "\n")


def _write_mtl(rng, path):
    names = [f"m{i}" for i in range(rng.integers(1, 5))]
    lines = []
    for nm in names:
        lines.append(f"newmtl {nm}")
        for key in ("Kd", "Ks", "Ke", "Kt"):
            if rng.random() < 0.6:
                lines.append(f"{key} " + " ".join(_num(rng, float(rng.random())) for _ in range(3)))
        for key, lo, hi in (("Ns", -5, 200), ("Ni", 0, 2.5), ("d", 0, 1), ("Tr", 0, 1), ("Pr", 0, 1)):
            if rng.random() < 0.4:
                lines.append(f"{key} {_num(rng, float(rng.uniform(lo, hi)))}")
        if rng.random() < 0.2:
            lines.append("map_Kd tex.png")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
    return names


def _write_scene(rng, d):
    names = _write_mtl(rng, os.path.join(d, "lib.mtl"))
    files = []
    for i in range(rng.integers(1, 4)):
        fn = f"mesh{i}.obj"
        _write_obj(rng, os.path.join(d, fn), names if rng.random() < 0.8 else [])
        files.append(fn)

    def v3():
        return ",".join(_num(rng, float(x)) for x in rng.normal(size=3) * 3)

    xml = [f'<Scene width="{rng.integers(64, 2000)}" maxRayDepth="{rng.integers(1, 9)}">']
    for _ in range(rng.integers(1, 7)):
        k = rng.integers(0, 6)
        if k == 0:
            xml.append(f'<Sphere position="{v3()}" radius="{_num(rng, float(rng.random()))}" diffuse="0.5,0.2,0.1"/>')
        elif k == 1:
            xml.append(f'<Rectangle position="{v3()}" u="{v3()}" v="{v3()}" rotation="{v3()}"/>')
        else:
            attrs = [f'file="{files[rng.integers(0, len(files))]}"', f'position="{v3()}"']
            if rng.random() < 0.5:
                attrs.append(f'scale="{_num(rng, float(rng.uniform(0.1, 3)))}"')
            if rng.random() < 0.5:
                attrs.append(f'rotation="{v3()}"')
            if rng.random() < 0.3:
                attrs += [f'basisX="{v3()}"', f'basisY="{v3()}"', f'basisZ="{v3()}"']
            if rng.random() < 0.3:
                attrs.append('diffuse="0.9,0.9,0.1"')
            if rng.random() < 0.4:
                attrs.append(f'clusterMaxTriangles="{rng.integers(1, 20)}"')
            if rng.random() < 0.3:
                attrs.append(f'clusterMaxExtent="{_num(rng, float(rng.uniform(0.2, 2)))}"')
            xml.append("<Mesh " + " ".join(attrs) + "/>")
    xml.append("</Scene>")
    path = os.path.join(d, "scene.xml")
    with open(path, "w") as f:
        f.write("\n".join(xml) + "\n")
    return path


@pytest.mark.parametrize("seed", range(40))
def test_random_scene_matches_reference_loader(nb, tmp_path, seed):
    from oracle import reference_ingest as ri

    if not ri.available():
        pytest.skip("oracle/_ref/libref_ingest.so not built")
    rng = np.random.default_rng(1000 + seed)
    path = _write_scene(rng, str(tmp_path))
    ref = ri.load_xml(path)
    mine = nb.load_scene_xml(path)
    assert ref is not None
    for k in ARRAYS:
        a, b = np.ascontiguousarray(getattr(mine, k)), np.ascontiguousarray(ref[k])
        assert a.size == b.size, k
        assert np.array_equal(a.reshape(b.shape).view(np.uint8), b.view(np.uint8)), k
    assert mine.settings == ref["settings"]
