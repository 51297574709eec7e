"""Seeded inputs for the shading pin: the contract oracle's shading functions and frames against the
reference's own (oracle/reference_shade.py, compiled from PathTracing.h / Scatter.h /
PathTraceKernel.metal). Used by tests/test_reference_pin.py and tests/golden/make_golden.py.

Uniforms are drawn on the 2^-24 grid the path tracer's Philox numbers lie on ((x >> 8) * 2^-24).
"""
import numpy as np

F32 = np.float32


def uniforms(rng, shape):
    return ((rng.integers(0, 2 ** 32, shape, dtype=np.uint64) >> 8).astype(F32) * F32(2.0 ** -24))


def unit(rng, n):
    v = rng.normal(size=(n, 3)).astype(F32)
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(F32)


def materials(rng, n):
    """Packed materials (5 float4, Material.h:32-44) over the ranges decodeMaterial clamps,
    including negative colours, opacity above 1 and transmissive / opaque mixes."""
    m = np.zeros((n, 20), F32)
    m[:, 0:3] = rng.uniform(-0.1, 1.0, (n, 3))
    m[:, 3] = rng.uniform(0.0, 1.2, n)
    m[:, 4:7] = rng.uniform(-0.1, 1.0, (n, 3))
    m[:, 7] = rng.uniform(0.0, 300.0, n)
    m[:, 8:11] = rng.uniform(-0.1, 2.0, (n, 3))
    m[:, 11] = rng.uniform(-1.0, 5.0, n)
    m[:, 12:15] = rng.uniform(-0.1, 1.0, (n, 3)) * (rng.random((n, 1)) < 0.5)
    m[:, 15] = rng.uniform(0.5, 2.5, n)
    m[:, 16:19] = -1.0
    m[:, 19] = rng.uniform(-0.2, 1.2, n)
    return m


def bsdf_cases(rng, n):
    """(materials, normal / view / light directions): the normal unnormalised, view and light on
    its side, plus 2 % of cases below the horizon."""
    nrm, v, l = unit(rng, n), unit(rng, n), unit(rng, n)
    v = np.where((np.sum(v * nrm, 1) < 0)[:, None], -v, v)
    l = np.where((np.sum(l * nrm, 1) < 0)[:, None], -l, l)
    flip = rng.random(n) < 0.02
    l[flip] = -l[flip]
    nvl = np.concatenate([nrm * rng.uniform(0.5, 2.0, (n, 1)), v, l], 1).astype(F32)
    return materials(rng, n), nvl


def light_cdf(rng, count=4096, sigma=1.5):
    cdf = np.cumsum(rng.lognormal(0.0, sigma, count)).astype(F32)
    xi = uniforms(rng, 10_000)
    xi[:4] = [0.0, F32(1.0 - 2.0 ** -24), 0.5, F32(2.0 ** -24)]
    return xi, cdf, float(cdf[-1])


def light_prims(rng, n):
    """Primitive records (7 float4) of spheres, triangles and rectangles (type in f4[0].w), some
    degenerate (zero radius, collinear vertices), and the two uniforms of each."""
    p = np.zeros((n, 28), F32)
    t = rng.integers(0, 3, n)
    p[:, 3] = t
    p[:, 0:3] = rng.uniform(-50, 50, (n, 3))
    p[:, 4:7] = rng.uniform(-5, 5, (n, 3))
    p[:, 8:11] = rng.uniform(-5, 5, (n, 3))
    p[t == 0, 4] = rng.uniform(-0.5, 3.0, (t == 0).sum())
    deg = (t == 1) & (rng.random(n) < 0.01)
    p[deg, 8:11] = p[deg, 4:7]
    return p, uniforms(rng, (n, 2))


def scatter_cases(rng, n):
    """Incoming direction, shading normal (facing the ray), front-face flag, material, 4 uniforms."""
    d, nn = -unit(rng, n), unit(rng, n)
    nn = np.where((np.sum(d * nn, 1) > 0)[:, None], -nn, nn)
    front = (rng.random(n) < 0.7).astype(np.uint8)
    return np.concatenate([d, nn], 1).astype(F32), front, materials(rng, n), uniforms(rng, (n, 4))


def reservoir_chains(rng, chains=2000, k=24):
    """Candidate streams for restirUpdateReservoir: light sample fields, pdfs (some <= 0), weight
    scales (some 0) and sample-count increments (some 0, some 3)."""
    n = chains * k
    c = np.zeros((n, 16), F32)
    c[:, 0:3] = rng.uniform(-10, 10, (n, 3))
    c[:, 3] = rng.integers(0, 1000, n)
    c[:, 4:7] = unit(rng, n)
    c[:, 7] = rng.uniform(0.01, 5.0, n)
    c[:, 8] = rng.uniform(-0.1, 3.0, n)
    c[:, 9:12] = rng.uniform(0.0, 2.0, (n, 3))
    c[:, 12] = rng.uniform(0.0, 1.0, n)
    c[:, 13] = rng.choice([1.0, 0.0, 0.5], n)
    c[:, 14] = rng.choice([1.0, 0.0, 3.0], n)
    return c, uniforms(rng, (chains, k))


# ------------------------------------------------------------------------------------------------
# Frames

def frame_scene(nb):
    """A small lit city: 8 emissive quads and 256 emissive triangles with lognormal power."""
    scene = nb.synth_city(seed=21, grid=6, size_m=200.0, target_tris=40_000, median_tris=600,
                          max_tris=8_000, emissive_quads=8, emissive_tris=256, emissive_sigma=1.5)
    return nb.SceneBVH(scene)


def nee_views(nb):
    """(view, tape seed) pairs: jittered pinhole views, one with 8 bounces (Russian roulette from
    bounce 5 on) and 2 spp, one with 3 bounces."""
    return [(nb.view_pinhole((0, 60, -180), (0, 10, 0), width=48, height=32, spp=2, max_depth=8, seed=3,
                             flags=nb.VIEW_CLAMP), 11),
            (nb.view_pinhole((80, 30, 20), (0, 5, 0), width=32, height=24, spp=1, max_depth=3, seed=4,
                             flags=nb.VIEW_CLAMP), 12)]


RESTIR_CANDIDATES = 16


def restir_views(nb, width=64, height=40):
    """Three frames of a slowly moving narrow camera (20 degrees), so that the reference's +-1 px
    neighbours and the reprojected pixel pass its surface gates on a good share of pixels."""
    out = []
    for f, pos in enumerate([(0, 60, -180), (0.5, 60, -179.5), (1.0, 59.8, -179)]):
        out.append((nb.view_pinhole(pos, (0, 10, 0), vfov=20.0, width=width, height=height, spp=1, max_depth=3,
                                    seed=3, frame=f, flags=nb.VIEW_RESTIR | nb.VIEW_CLAMP), 100 + f))
    return out


def tapes(seed, pixels, length=1024):
    return uniforms(np.random.default_rng(seed), (pixels, length))


def pixel_rel(a, b):
    """Per pixel: L1 difference over L1 of the reference, floored at 1e-3 (dark pixels)."""
    return np.abs(a - b).sum(1) / np.maximum(np.abs(a).sum(1), 1e-3)


# ------------------------------------------------------------------------------------------------
# Reference outputs: computed live from oracle/_ref/libref_shade.so, or read from the golden file
# tests/golden/shading_ref.npz that tests/golden/make_golden.py writes with the same code. The
# golden keeps the first GOLDEN_CASES cases of each ulp-level function, sha256 digests of the
# bit-exact ones, and the frames.

GOLDEN_CASES = 2000
GOLDEN_FILE = "shading_ref.npz"


def function_inputs():
    rng = np.random.default_rng(2024)
    d = {"mats": materials(rng, 10_000)}
    d["xi"], d["cdf"], d["total"] = light_cdf(rng)
    d["cand"], d["cxi"] = reservoir_chains(rng)
    d["bmats"], d["nvl"] = bsdf_cases(rng, 10_000)
    d["prims"], d["uv"] = light_prims(rng, 12_000)
    d["dn"], d["front"], d["smats"], d["tape4"] = scatter_cases(rng, 10_000)
    return d


def sha(*arrays):
    import hashlib

    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
    return h.hexdigest()


def reference_function_outputs(rs, d):
    """Every reference function on the full inputs."""
    out = {"decode_1": rs.decode_material(d["mats"], 1.0)[:, :17], "decode_073": rs.decode_material(d["mats"], 0.73)[:, :17]}
    out["sel_off"], out["sel_pdf"] = rs.select_light(d["xi"], d["cdf"], d["total"])
    out["resv"] = rs.reservoir_chain(d["cand"], d["cxi"])
    out["bsdf"] = rs.bsdf(d["bmats"], d["nvl"])
    out["lp"], out["lp_ok"] = rs.sample_light_point(d["prims"], d["uv"])
    out["sc_dir"], out["sc_w"], out["sc_draws"] = rs.scatter(d["dn"], d["front"], d["smats"], d["tape4"])
    return out


def golden_function_outputs(full):
    g = {k + "_sha": np.array(sha(full[k])) for k in ("decode_1", "decode_073", "sel_off", "sel_pdf", "resv")}
    for k in ("bsdf", "lp", "lp_ok", "sc_dir", "sc_w", "sc_draws"):
        g[k] = full[k][:GOLDEN_CASES]
    return g


def reference_frames(nb, orc, rs):
    """The reference's frames: the path-traced views and the ReSTIR reference-mode sequence."""
    sb = frame_scene(nb)
    os_ = orc.OracleScene(sb)
    lights = orc.light_tables(os_, sb.materials)
    out = {}
    for i, (view, seed) in enumerate(nee_views(nb)):
        w, h = int(view["width"][0]), int(view["height"][0])
        out[f"nee{i}_rgb"], _ = rs.render_frame(os_, sb.materials, view, lights, tapes(seed, w * h))
    prev_v, prev_tex = None, None
    for f, (view, seed) in enumerate(restir_views(nb)):
        w, h = int(view["width"][0]), int(view["height"][0])
        a, tex = rs.render_frame(os_, sb.materials, view, lights, tapes(seed, w * h),
                                 restir=(1, RESTIR_CANDIDATES, 1), prev_view=prev_v, prev_tex=prev_tex)
        out[f"restir{f}_rgb"], out[f"restir{f}_tex"] = a, tex
        prev_v, prev_tex = view, tex
    return out


def golden_frames(full):
    g = {}
    for k, v in full.items():
        if k.endswith("_tex"):
            f = k[: -len("_tex")]
            g[f + "_count"] = v[2][:, 2].astype(np.uint16)           # sample counts
            g[f + "_light"] = np.where(v[2][:, 1] > 0, v[0][:, 3], -1).astype(np.int32)
            g[f + "_surf_sha"] = np.array(sha(v[3]))
        else:
            g[k] = v
    return g
