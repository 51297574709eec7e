"""Pins the oracle and the builder to the reference's own code.

The reference ships no golden vectors for this path, so the fixtures in tests/golden/ were
made by running the reference's own SceneBVH.cpp / Scene.cpp builder and its MSL traversal
(PathTracing.h firstHitTLAS, compiled as C++ through a Metal-compatibility header) here; see
tests/golden/make_golden.py. Where oracle/_ref is built, the same checks also run live.

The contract differs from the reference traversal in three documented ways, and every
differing ray must be explained by one of them:
  * the reference ignores tmax (firstHitTLAS never reads ray.maxDistance);
  * exact tie in t: the contract returns the lower primitive index;
  * near tie: the reference's exact per-BLAS pruning skipped a primitive whose hit is nearer by
    a few ulps (its box entry rounded past the current best); the contract returns that nearer
    primitive.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from tests import raysets

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def _scene(nb, name):
    if name == "ico":
        return nb.synth_icospheres(seed=11, instances=64, extent=100.0)
    return nb.synth_city(seed=5, grid=8, size_m=250.0, target_tris=120_000, median_tris=1000,
                         max_tris=20_000, emissive_quads=8)


def _golden_rays(sb, seed):
    return np.concatenate([raysets.aimed_rays(sb, 3000, seed), raysets.random_rays(sb, 1000, seed + 1),
                           raysets.edge_case_rays(sb, seed + 2)])


def classify(rays, h_ref, h_con):
    """Counts of each explained difference; raises on an unexplained one."""
    r = np.ascontiguousarray(h_ref).view(np.int32).reshape(-1, 5)
    c = np.ascontiguousarray(h_con).view(np.int32).reshape(-1, 5)
    diff = np.nonzero((r != c).any(1))[0]
    tr, tc = h_ref["t"][diff], h_con["t"][diff]
    pr, pc = h_ref["prim"][diff], h_con["prim"][diff]
    finite_tmax = np.isfinite(rays["tmax"][diff])
    tie = (~finite_tmax) & (pc >= 0) & (tc == tr) & (pc < pr)
    near = (~finite_tmax) & (pc >= 0) & (pr >= 0) & (tc < tr) & (tr - tc <= tr * np.float32(2.0 ** -10))
    bad = ~(finite_tmax | tie | near)
    assert not bad.any(), (f"{bad.sum()} unexplained differences, e.g. rays {diff[bad][:5]}: "
                           f"ref {h_ref[diff[bad][:3]]} contract {h_con[diff[bad][:3]]}")
    return {"differ": int(diff.size), "tmax_ignored": int(finite_tmax.sum()), "exact_tie": int(tie.sum()),
            "near_tie": int(near.sum())}


@pytest.mark.parametrize("name", ["ico", "city"])
def test_builder_matches_reference_golden(nb, name):
    want = json.load(open(os.path.join(GOLD, "scenebvh_sha256.json")))[name]
    sb = nb.SceneBVH(_scene(nb, name))
    got = {"bvh_nodes": _sha(sb.bvh_nodes), "tlas_nodes": _sha(sb.tlas_nodes), "prims": _sha(sb.prims),
           "materials": _sha(sb.materials), "prim_indices": _sha(sb.prim_indices),
           "blas_root": _sha(np.ascontiguousarray(sb.instances["blas_root_index"], np.int32))}
    assert got == want


@pytest.mark.parametrize("name", ["ico", "city"])
def test_oracle_against_reference_golden(nb, orc, name):
    g = np.load(os.path.join(GOLD, f"hits_{name}.npz"))
    sb = nb.SceneBVH(_scene(nb, name))
    rays = _golden_rays(sb, 1000)
    assert str(g["ray_sha"]) == _sha(rays)
    h_ref = g["ref"].view(orc.HIT_DTYPE).reshape(-1)
    h_con = orc.OracleScene(sb).closest(rays)
    assert np.array_equal(np.ascontiguousarray(h_con).view(np.int32).reshape(-1), g["contract"].reshape(-1))
    stats = classify(rays, h_ref, h_con)
    inf = np.isinf(rays["tmax"])
    # the reference and the contract agree on the overwhelming majority of unbounded rays
    assert stats["exact_tie"] + stats["near_tie"] < 0.03 * inf.sum(), stats


def test_reference_live(nb, orc):
    from oracle import reference as ref

    if not ref.available():
        pytest.skip("reference build (oracle/_ref) not present")
    scene = nb.synth_city(seed=77, grid=6, size_m=200.0, target_tris=60_000, median_tris=800,
                          max_tris=10_000, emissive_quads=4)
    r = ref.build_scene(scene)
    sb = nb.SceneBVH(scene)
    for k in ("bvh_nodes", "tlas_nodes", "prims", "materials", "prim_indices"):
        assert np.array_equal(getattr(sb, k).view(np.uint32), r[k].view(np.uint32)), k
    cam = nb.Camera((0, 50, -150), (0, 0, 0), width=200, height=120)
    prim = cam.primary_rays(1, seed=3)
    rays = np.concatenate([prim, _golden_rays(sb, 4242)])
    h_con = orc.OracleScene(sb).closest(rays)
    classify(rays, ref.closest(sb, rays), h_con)
    # with some objects evicted and primitives deactivated
    rng = np.random.default_rng(2)
    active = (rng.random(sb.prim_count) > 0.15).astype(np.uint8)
    root = sb.instances["blas_root_index"].copy()
    root[rng.random(sb.object_count) < 0.25] = -1
    classify(rays, ref.closest(sb, rays, active=active, blas_root=root),
             orc.OracleScene(sb, active=active, blas_root=root).closest(rays))


# ---------------------------------------------------------------------------------------------
# Shading pin: the oracle's path tracer and ReSTIR (oracle/pathtrace.cpp, the checker of the CUDA
# path tracer) against the reference's own shading code (oracle/ref/ref_shade.cpp: PathTracing.h,
# Scatter.h and PathTraceKernel.metal compiled as C++), function by function and frame by frame,
# on identical inputs and identical random numbers ("tapes", drawn in the reference's order).
#
# Where the two are not bit-identical the difference is one of these, each isolated below:
#   * contract difference 6 (pt_math: x^5 as a product, sin/cos(2 pi u) and pow(u, e) by fixed
#     series) and the host build of the MSL evaluating pi * denom^2 and 4 pi r^2 in double (M_PI is
#     a double literal in C++): ulp-level;
#   * contract difference 4 (light visibility as an any-hit over (1e-4, dist - eps) rather than the
#     reference's closest hit accepted when it is the light at t >= dist - eps) and the temporal
#     reprojection (the previous view's ray-plane intersection rather than a float matrix): the
#     oracle's reference rules (oracle.set_reference_rules) switch both to the reference's, and the
#     frames then agree pixel for pixel.
from tests import shading_pin as sp  # noqa: E402


def _rs():
    from oracle import reference_shade as rs

    if not rs.available():
        pytest.skip("reference shading build (oracle/_ref/libref_shade.so) not present")
    return rs


def _bits_equal(a, b):
    a, b = np.ascontiguousarray(a, np.float32), np.ascontiguousarray(b, np.float32)
    return (a.view(np.uint32) == b.view(np.uint32)).reshape(a.shape[0], -1).all(1)


def _ulps(a, b):
    ia = np.ascontiguousarray(a, np.float32).view(np.int32).astype(np.int64)
    ib = np.ascontiguousarray(b, np.float32).view(np.int32).astype(np.int64)
    ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
    ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
    return np.abs(ia - ib)


def _libm_powf():
    import ctypes

    lm = ctypes.CDLL("libm.so.6")
    lm.powf.restype, lm.powf.argtypes = ctypes.c_float, [ctypes.c_float, ctypes.c_float]
    return lambda x, e: np.array([lm.powf(float(t), e) for t in x], np.float32)


def bsdf_model(dec, nvl, reference):
    """evaluateDirectLightingBsdf (PathTracing.h:249-293) in float32 numpy, in the operation order
    both implementations use. reference=True: pi * denom^2 in double and x^5 by libm powf, as the
    reference's host build computes them; False: in float and by products (contract difference 6)."""
    F = np.float32

    def dot(a, b):
        return (a[:, 0] * b[:, 0] + a[:, 1] * b[:, 1]) + a[:, 2] * b[:, 2]

    def nrm(a):
        return a / np.sqrt(dot(a, a))[:, None]

    with np.errstate(all="ignore"):
        n, v, l = nrm(nvl[:, 0:3]), nrm(nvl[:, 3:6]), nrm(nvl[:, 6:9])
        ok = np.isfinite(n).all(1) & np.isfinite(v).all(1) & np.isfinite(l).all(1)
        nl, nv = np.maximum(dot(n, l), F(0)), np.maximum(dot(n, v), F(0))
        ok &= (nl > 0) & (nv > 0)
        dc = np.maximum(dec[:, 0:3], F(0)) * dec[:, 3:4]
        sc = np.clip(dec[:, 4:7] * dec[:, 3:4], F(0), F(1))
        r = np.clip(dec[:, 16], F(0), F(1))
        alpha = np.maximum(r * r, F(0.001))
        a2 = alpha * alpha
        h = nrm(v + l)
        nh, vh = np.maximum(dot(n, h), F(0)), np.maximum(dot(v, h), F(0))
        den = nh * nh * (a2 - F(1)) + F(1)
        if reference:
            pd = (np.float64(np.pi) * den.astype(np.float64) * den.astype(np.float64)).astype(F)
        else:
            pd = F(np.pi) * den * den
        D = a2 / np.maximum(pd, F(1e-4))
        k = alpha + F(1)
        k = (k * k) / F(8)
        G = (nv / (nv * (F(1) - k) + k)) * (nl / (nl * (F(1) - k) + k))
        x = np.maximum(F(1) - vh, F(0))
        Fc = _libm_powf()(x, 5.0) if reference else (x * x) * (x * x) * x
        Fr = sc + (F(1) - sc) * Fc[:, None]
        out = dc / F(np.pi) + (Fr * (D * G)[:, None]) / np.maximum(F(4) * nl * nv, F(1e-4))[:, None]
    out[~ok] = 0
    return out.astype(F)


def _resv_canonical(a, reference):
    """Reservoir chain outputs in one form: slot 7 = 1 / area (the oracle stores that, the
    reference the area) where the reservoir is valid, else 0."""
    a = np.array(a, np.float32)
    valid = a[:, 15] > 0
    inv = np.float32(1) / np.where(valid, a[:, 7], np.float32(1)) if reference else a[:, 7]
    a[:, 7] = np.where(valid, inv, np.float32(0))
    return a


def _gold(name):
    return np.load(os.path.join(GOLD, name), allow_pickle=False)


@pytest.fixture(scope="module", params=["live", "golden"])
def function_refs(request):
    """(inputs, reference outputs): live from oracle/_ref, or the committed golden (first
    GOLDEN_CASES cases of the ulp-level functions, digests of the bit-exact ones)."""
    d = sp.function_inputs()
    if request.param == "live":
        full = sp.reference_function_outputs(_rs(), d)
        full["resv"] = _resv_canonical(full["resv"], True)
        g = sp.golden_function_outputs(full)
        g.update({k: full[k] for k in ("bsdf", "lp", "lp_ok", "sc_dir", "sc_w", "sc_draws")})
        return d, g
    g = dict(_gold(sp.GOLDEN_FILE))
    return d, g


def test_shading_functions_pinned(orc, function_refs):
    """>= 10^4 seeded cases per function against the reference's own functions (live; the golden
    holds digests of all cases of the bit-exact ones and the first 2,000 of the others)."""
    d, g = function_refs
    # decodeMaterial, selectLightOffset / lightPdfFromCdf (xi = 0 and just below 1 included) and
    # restirUpdateReservoir chains with restirContribution / restirTargetFromCandidate weights:
    # bit for bit
    assert sp.sha(orc.decode_material(d["mats"], 1.0)) == str(g["decode_1_sha"])
    assert sp.sha(orc.decode_material(d["mats"], 0.73)) == str(g["decode_073_sha"])
    off, pdf = orc.select_light(d["xi"], d["cdf"], d["total"])
    assert sp.sha(off) == str(g["sel_off_sha"]) and sp.sha(pdf) == str(g["sel_pdf_sha"])
    resv = _resv_canonical(orc.reservoir_chain(d["cand"], d["cxi"]), False)
    assert sp.sha(resv) == str(g["resv_sha"])
    assert (resv[:, 15] > 0).mean() > 0.5 and (resv[:, 16] < d["cxi"].shape[1]).mean() > 0.5
    # evaluateDirectLightingBsdf: each side is reproduced bit for bit by one float32 model, so the
    # named terms (pi * denom^2 in double, x^5 by powf) explain every difference; <= 8 ulp apart
    n = g["bsdf"].shape[0]
    mats, nvl = d["bmats"][:n], d["nvl"][:n]
    dec = orc.decode_material(mats)
    ra, ob = g["bsdf"], orc.bsdf(mats, nvl)
    assert _bits_equal(ra, bsdf_model(dec, nvl, True)).all()
    assert _bits_equal(ob, bsdf_model(dec, nvl, False)).all()
    assert _ulps(ra, ob).max() <= 8 and _bits_equal(ra, ob).mean() > 0.75
    # sampleLightPoint: triangles and rectangles bit for bit; spheres (sin/cos by series, area in
    # double) within 1e-6 relative; the same samples rejected (zero radius, collinear vertices)
    n = g["lp"].shape[0]
    prims = d["prims"][:n]
    pa, ka = g["lp"], g["lp_ok"]
    pb, kb = orc.sample_light_point(prims, d["uv"][:n])
    assert np.array_equal(ka, kb) and 0 < ka.mean() < 1
    t = prims[:, 3].astype(int)
    assert _bits_equal(pa[(t > 0) & (ka == 1)], pb[(t > 0) & (kb == 1)]).all()
    sph = (t == 0) & (ka == 1)
    assert np.allclose(pa[sph], pb[sph], rtol=1e-6, atol=1e-6)
    # scatter (cosine lobe / Phong lobe / dielectric): the same lobes and draws, the weights bit for
    # bit, the directions per lobe
    n = g["sc_dir"].shape[0]
    dn, front, smats, tape4 = d["dn"][:n], d["front"][:n], d["smats"][:n], d["tape4"][:n]
    da, wa, ka = g["sc_dir"], g["sc_w"], g["sc_draws"]
    db, wb, kb = orc.scatter(dn, front, smats, tape4)
    assert np.array_equal(ka, kb) and set(np.unique(ka)) >= {2, 3}  # dielectric 2, the lobes 3
    assert _bits_equal(wa, wb).all()
    # lobe of each case as scatter picks it (Scatter.h:78-99), from the decoded material
    dec = orc.decode_material(smats)

    def lum(c):
        return c[:, 0] * np.float32(0.2126) + c[:, 1] * np.float32(0.7152) + c[:, 2] * np.float32(0.0722)

    dw = np.maximum(lum(dec[:, 0:3]) * dec[:, 3], 0)
    tw = np.maximum(lum(dec[:, 12:15]) * (1 - dec[:, 3]), 0)
    sw = np.where(tw > 0, 0, np.maximum(lum(dec[:, 4:7]) * dec[:, 3], 0))
    xi = tape4[:, 0] * (dw + sw + tw)
    lobe = np.where(xi < dw, 0, np.where(xi - dw < sw, 1, 2))
    err = np.abs(da - db).max(1)
    assert min((lobe == k).sum() for k in range(3)) > 100
    assert _bits_equal(da[lobe == 2], db[lobe == 2]).all()  # dielectric: reflect / refract, no series
    assert err[lobe == 0].max() < 1e-6  # cosine lobe: sin / cos(2 pi u) by series
    # Phong lobe: cos theta = u^(1 / (e + 1)) by series; sin theta = sqrt(1 - cos^2) magnifies its
    # last-bit difference where cos theta is near 1
    assert err[lobe == 1].max() < 2e-4 and err[lobe == 1].mean() < 5e-6


@pytest.fixture(scope="module", params=["live", "golden"])
def frame_refs(request, nb, orc):
    if request.param == "live":
        return sp.golden_frames(sp.reference_frames(nb, orc, _rs()))
    return dict(_gold(sp.GOLDEN_FILE))


def _oracle_frame(nb, orc, view, seed, rules):
    sb = sp.frame_scene(nb)
    os_ = orc.OracleScene(sb)
    w, h = int(view["width"][0]), int(view["height"][0])
    orc.set_reference_rules(rules, track=True)
    try:
        b = orc.render_tape(os_, sb.materials, view, sp.tapes(seed, w * h))
        counts = orc.set_reference_rules(0)
    finally:
        orc.set_reference_rules(0)
    return b, counts


@pytest.mark.parametrize("rules", [0, 1])
def test_path_tracer_frames_pinned(nb, orc, frame_refs, rules):
    """pathTraceKernel + rayColor (raygen, sky, emission, one-sample NEE, scatter, Russian
    roulette, clamps) against the oracle's path tracer on the same tapes: every pixel within 1e-4
    (the contract's radiance bar), most bit for bit, under the contract's visibility (rules=0) and
    the reference's (rules=1)."""
    for i, (view, seed) in enumerate(sp.nee_views(nb)):
        a = frame_refs[f"nee{i}_rgb"]
        b, (tests, differ) = _oracle_frame(nb, orc, view, seed, rules)
        rel = sp.pixel_rel(a, b)
        assert rel.max() < 1e-4 and rel.mean() < 1e-6, (rel.max(), rel.mean())
        assert _bits_equal(a, b).mean() > 0.4
        assert tests > 500 and differ <= 1e-3 * tests, (tests, differ)


def _oracle_restir(nb, orc, rules):
    sb = sp.frame_scene(nb)
    ro = orc.RestirOracle(orc.OracleScene(sb), sb.materials, candidates=sp.RESTIR_CANDIDATES, temporal=True,
                          reference_mode=True)
    out = []
    orc.set_reference_rules(rules, track=True)
    try:
        for view, seed in sp.restir_views(nb):
            w, h = int(view["width"][0]), int(view["height"][0])
            b, _ = ro.render(view, sp.tapes(seed, w * h))
            resv, surf = ro.last
            out.append((b, resv.copy(), surf.copy(), orc.set_reference_rules(rules, track=True)))
    finally:
        orc.set_reference_rules(0)
    return out


def test_restir_reference_mode_pinned(nb, orc, frame_refs):
    """The oracle's ReSTIR reference mode against the reference's own rayColor ReSTIR over three
    frames of a moving camera (candidates with per-candidate visibility, previous-frame +-1 px
    spatial and reprojected temporal reuse, MIS weights, Jacobian clamp, reservoir and surface
    textures), under the reference's rules: every pixel within 1e-4, the same selected light and
    sample count in every reservoir, the surface records bit for bit."""
    seq = _oracle_restir(nb, orc, orc.RULE_VISIBILITY | orc.RULE_REPROJECTION)
    for f, (b, resv, surf, _) in enumerate(seq):
        a = frame_refs[f"restir{f}_rgb"]
        rel = sp.pixel_rel(a, b)
        assert rel.max() < 1e-4, (f, rel.max(), np.argmax(rel))
        light = np.where(resv[:, 3].view(np.int32) >= 0, resv[:, 3].view(np.int32), -1)
        assert np.array_equal(frame_refs[f"restir{f}_light"], light)
        count = frame_refs[f"restir{f}_count"]
        assert np.array_equal(count, resv[:, 10].astype(np.uint16))
        assert str(frame_refs[f"restir{f}_surf_sha"]) == sp.sha(np.ascontiguousarray(surf[:, 0:4]))
        if f > 0:  # reuse is exercised: reservoirs with more samples than the candidates
            assert (count > sp.RESTIR_CANDIDATES).mean() > 0.05


def test_restir_reference_mode_contract_rules(nb, orc, frame_refs):
    """The same sequence under the contract's rules (what the CUDA path computes). The pixels that
    differ are those whose light-visibility decision the two rules take differently (about 1 in
    20,000 here), or that reuse such a pixel's reservoir; one flipped decision can move its pixel
    by a whole light sample, so the bound is on how many pixels differ, not on how much."""
    seen = 0
    for f, (b, resv, surf, (tests, differ)) in enumerate(_oracle_restir(nb, orc, 0)):
        a = frame_refs[f"restir{f}_rgb"]
        rel = sp.pixel_rel(a, b)
        seen += differ
        assert differ <= 1e-4 * tests, (f, tests, differ)
        assert (rel > 1e-4).sum() <= 4 * seen, (f, (rel > 1e-4).sum(), seen)
        assert np.abs(a - b).sum() / np.abs(a).sum() < 1e-3
