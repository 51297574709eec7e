// ORACLE glue — test infrastructure only. Runs the reference's own shading code on the host
// cores: pathTraceKernel (Renderer/Shaders/PathTraceKernel.metal) with its raygen, rayColor bounce
// loop, one-sample NEE, ReSTIR DI (candidates, previous-frame spatial and temporal reuse with its
// MIS weights and Jacobian), decodeMaterial, evaluateDirectLightingBsdf, selectLightOffset /
// lightPdfFromCdf, sampleLightPoint and scatter (PathTracing.h, Scatter.h), compiled as C++
// through shim/metal_compat.h. None of the reference's code is changed.
//
// Random numbers. The reference draws u = randomFloat(seed) and advances seed = random(seed)
// (Random.h:6-17), starting each pixel from a hash of its uv (PathTraceKernel.metal:67-68). Here
// Random.h is replaced: a seed is a position in a list of uniforms supplied by the caller (a
// "tape"), randomFloat(seed) reads that position (0.5 past the end) and random(seed) = seed + 1;
// the per-pixel hash returns 0, so every pixel starts at the head of its own tape. The contract
// oracle's path tracer can draw from the same tape in the same order (oracle/pathtrace.cpp,
// Draws), so both run on identical numbers.
//
// Inputs the reference computes on the host (Renderer.cpp) and that cannot be compiled here (it
// needs Metal) are passed in: the light tables (indices, CDF, per-primitive pdf,
// Renderer.cpp:5161-5211), the instance records (:5293-5358, rebuilt as ref_trace.cpp does) and
// the previous frame's view-projection matrix, built below from the previous pinhole view.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../view_projection.h"
#include "metal_compat.h"
using namespace metal;

#define RANDOM_H  // Random.h is replaced by the tape below
namespace tape {
thread_local const float *values = nullptr;
thread_local uint32_t length = 0;
}  // namespace tape
inline uint32_t random(uint32_t s) { return s + 1u; }
inline float randomFloat(uint32_t s) { return s < tape::length ? tape::values[s] : 0.5f; }
inline float random(float2, float3) { return 0.0f; }

#define kernel
#include "PathTraceKernel.metal"
#undef kernel
#undef thread
#undef device
#undef constant

namespace {

// nomad_view (include/nomad_rt.h): pinhole camera as populateViewportUniforms fills it.
struct ViewIn {
  float cam[3], vu[3], vv[3], fp[3];
  uint32_t w, h, spp, maxDepth, seedLo, seedHi, frame, flags;
};

float3 f3(const float *p) { return float3(p[0], p[1], p[2]); }

// The previous frame's view-projection matrix, built from the previous pinhole view so that its
// NDC follows the pixel rows (oracle/view_projection.h). The reference's own matrix
// (Renderer.cpp:6972-6989, makePerspectiveMatrix / makeViewMatrix :1374-1416) has NDC y pointing
// up while its raygen numbers rows from the top (populateViewportUniforms :1237-1259), so
// rayColor's temporal source (PathTracing.h:1436-1445) would be the vertically mirrored pixel.
float4x4 prev_view_projection(const ViewIn &v) {
  float m[16];
  oracle_vp::build(v.cam, v.vu, v.vv, v.fp, m);
  float4x4 r;
  for (int c = 0; c < 4; ++c) r.columns[c] = float4(m[4 * c], m[4 * c + 1], m[4 * c + 2], m[4 * c + 3]);
  return r;
}

template <typename F> void parallel(uint64_t n, uint32_t threads, F fn) {
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        uint64_t b = next.fetch_add(16);
        if (b >= n) break;
        for (uint64_t i = b; i < std::min(n, b + 16); ++i) fn(i);
      }
    });
  for (auto &t : pool) t.join();
}

void set_tape(const float *t, uint32_t len) {
  tape::values = t;
  tape::length = len;
}

}  // namespace

extern "C" {

// One frame of the reference's pathTraceKernel over every pixel of `view`.
//   restir: {enabled, candidate count, temporal reuse}; prev_view (null on the first frame) and
//   prev_tex hold the previous frame's view and its ReSTIR textures, out_tex receives this
//   frame's: per pixel 5 float4 = data0 (light position, id), data1 (light normal, area),
//   data2 (pdf, weight sum, sample count, selected weight), surface position (xyz, depth),
//   surface normal.
//   tapes: tape_len uniforms per pixel. out_rgb: 3 floats per pixel (the clamped average).
int ref_render_frame(const float *bvh, uint32_t bvh_count, const float *tlas, uint32_t tlas_count,
                     const float *prims, const float *materials, const int32_t *prim_indices,
                     const uint8_t *active, const int32_t *blas_root, const int32_t *prim_object,
                     uint32_t prim_count, const uint32_t *light_idx, const float *light_cdf,
                     uint32_t light_count, float light_total, const float *light_pdf, const void *view,
                     const void *prev_view, const uint32_t *restir, const float *prev_tex, float *out_tex,
                     const float *tapes, uint32_t tape_len, float *out_rgb, uint32_t threads) {
  if (!bvh || !tlas || !prims || !materials || !prim_indices || !active || !blas_root || !prim_object || !view ||
      !restir || !tapes || !out_rgb || (restir[0] && !out_tex))
    return 1;
  const ViewIn &v = *static_cast<const ViewIn *>(view);
  uint32_t objCount = 0;
  for (uint32_t p = 0; p < prim_count; ++p) objCount = std::max<uint32_t>(objCount, prim_object[p] + 1);
  std::vector<InstanceRecord> inst(objCount);
  for (uint32_t o = 0; o < objCount; ++o) inst[o] = InstanceRecord{blas_root[o], 0u, 0u, 0u};
  for (uint32_t p = prim_count; p-- > 0;) {
    InstanceRecord &r = inst[prim_object[p]];
    r.primitiveBase = p;
    r.primitiveIndexBase = p;
    r.primitiveCount += 1;
  }
  std::vector<uint32_t> remap(prim_count);
  for (uint32_t p = 0; p < prim_count; ++p) remap[p] = p;
  std::vector<std::atomic<uint32_t>> stats(2ull * prim_count + 2);
  std::vector<float> nopdf(prim_count, 0.0f);

  UniformsData u{};
  u.cameraPosition = f3(v.cam);
  u.screenSize = float2((float)v.w, (float)v.h);
  u.aperture = 0.0f;
  u.focusDistance = 1.0f;
  u.viewportU = f3(v.vu);
  u.viewportV = f3(v.vv);
  u.firstPixelPosition = f3(v.fp);
  u.rayDx = u.viewportU / (float)v.w;  // populateViewportUniforms, Renderer.cpp:1256-1257
  u.rayDy = u.viewportV / (float)v.h;
  u.randomSeed = float3(0.0f);
  u.primitiveCount = prim_count;
  u.triangleCount = prim_count;
  u.totalPrimitiveCount = prim_count;
  u.tlasNodeCount = tlas_count;
  u.blasNodeCount = bvh_count;
  u.maxRayDepth = v.maxDepth;
  u.debugAS = 0;
  u.lightCount = light_count;
  u.lightTotalWeight = light_total;
  u.minSamplesPerPixel = v.spp;
  u.maxSamplesPerPixel = v.spp;
  u.textureCount = 0;
  u.environmentMapEnabled = 0;
  u.environmentMapIntensity = 0.0f;
  u.restirEnabled = restir[0];
  u.restirCandidateCount = restir[1];
  u.restirTemporalReuse = restir[2];
  u.cameraMotionMetric = 0.0f;
  u.prevViewProjection = prev_view ? prev_view_projection(*static_cast<const ViewIn *>(prev_view)) : float4x4{};

  const uint32_t W = v.w, H = v.h;
  std::vector<float4> rgb(W * H), alb(W * H), nrm(W * H), pos(W * H);
  auto tex = [&](float4 *d, uint32_t w, uint32_t h) {
    texture2d<float, access::write> t;
    t.data = d, t.w = w, t.h = h;
    return t;
  };
  // ReSTIR textures: planes of W*H float4 each
  std::vector<float4> outPlanes(restir[0] ? 5ull * W * H : 1), prevPlanes;
  const bool havePrev = restir[0] && prev_view && prev_tex;
  if (havePrev) prevPlanes.assign(reinterpret_cast<const float4 *>(prev_tex),
                                  reinterpret_cast<const float4 *>(prev_tex) + 5ull * W * H);
  auto outTex = [&](int k) { return restir[0] ? tex(outPlanes.data() + (size_t)k * W * H, W, H) : tex(nullptr, 0, 0); };
  auto prevTex = [&](int k) {
    texture2d<float, access::read> t;
    if (havePrev) t.data = prevPlanes.data() + (size_t)k * W * H, t.w = W, t.h = H;
    return t;
  };
  array<texture2d<float, access::sample>, kMaxMaterialTextures> materialTextures{};
  texture2d<float, access::sample> env;
  sampler envSampler;
  TileRegion tile{uint2(0u, 0u), uint2(W, H)};
  const float4 *B = reinterpret_cast<const float4 *>(bvh);
  const float4 *T = reinterpret_cast<const float4 *>(tlas);
  const float4 *P = reinterpret_cast<const float4 *>(prims);
  const float4 *M = reinterpret_cast<const float4 *>(materials);
  auto c0 = tex(rgb.data(), W, H), c1 = tex(alb.data(), W, H), c2 = tex(nrm.data(), W, H), c3 = tex(pos.data(), W, H);
  auto o0 = outTex(0), o1 = outTex(1), o2 = outTex(2), o3 = outTex(3), o4 = outTex(4);
  auto p0 = prevTex(0), p1 = prevTex(1), p2 = prevTex(2), p3 = prevTex(3), p4 = prevTex(4);
  parallel((uint64_t)W * H, threads, [&](uint64_t i) {
    set_tape(tapes + i * tape_len, tape_len);
    uint2 gid((uint)(i % W), (uint)(i / W));
    pathTraceKernel(B, P, M, &u, nullptr, nullptr, prim_indices, T, active, light_idx, light_cdf,
                    light_pdf ? light_pdf : nopdf.data(), remap.data(), stats.data(), inst.data(), nullptr,
                    c0, c1, c2, c3, o0, o1, o2, p0, p1, p2, o3, o4, p3, p4, materialTextures, env, envSampler, tile,
                    gid);
  });
  for (uint64_t i = 0; i < (uint64_t)W * H; ++i) {
    out_rgb[3 * i] = rgb[i].x;
    out_rgb[3 * i + 1] = rgb[i].y;
    out_rgb[3 * i + 2] = rgb[i].z;
  }
  if (restir[0]) std::memcpy(out_tex, outPlanes.data(), sizeof(float4) * 5ull * W * H);
  return 0;
}

// decodeMaterial (PathTracing.h:165-196) of n packed materials (5 float4 each): per material 20
// floats = diffuse xyz, opacity, specular xyz, shininess, emission xyz, power, transmission xyz,
// index of refraction, roughness, diffuse / specular / normal texture index.
void ref_decode_material(const float *mats, uint32_t n, float lod, float *out) {
  const float4 *M = reinterpret_cast<const float4 *>(mats);
  for (uint32_t i = 0; i < n; ++i) {
    MaterialPayload m = decodeMaterial(int(i * kMaterialFloat4Count), M, lod);
    float *o = out + 20ull * i;
    const float vals[20] = {m.diffuseColor.x, m.diffuseColor.y, m.diffuseColor.z, m.opacity,
                            m.specularColor.x, m.specularColor.y, m.specularColor.z, m.shininess,
                            m.emissionColor.x, m.emissionColor.y, m.emissionColor.z, m.emissionPower,
                            m.transmissionColor.x, m.transmissionColor.y, m.transmissionColor.z,
                            m.indexOfRefraction, m.roughness, (float)m.diffuseTextureIndex,
                            (float)m.specularTextureIndex, (float)m.normalTextureIndex};
    std::memcpy(o, vals, sizeof(vals));
  }
}

// evaluateDirectLightingBsdf (:249-293) of decodeMaterial(material i, lod 1) for normal, view
// and light directions nvl[9 i .. 9 i + 8]; 3 floats per case.
void ref_bsdf(const float *mats, const float *nvl, uint32_t n, float *out) {
  const float4 *M = reinterpret_cast<const float4 *>(mats);
  for (uint32_t i = 0; i < n; ++i) {
    MaterialPayload m = decodeMaterial(int(i * kMaterialFloat4Count), M, 1.0f);
    const float *q = nvl + 9ull * i;
    float3 f = evaluateDirectLightingBsdf(m, f3(q), f3(q + 3), f3(q + 6));
    out[3 * i] = f.x, out[3 * i + 1] = f.y, out[3 * i + 2] = f.z;
  }
}

// selectLightOffset / lightPdfFromCdf (:219-247) for each xi.
void ref_select_light(const float *xi, uint32_t n, const float *cdf, uint32_t count, float total, uint32_t *off,
                      float *pdf) {
  for (uint32_t i = 0; i < n; ++i) {
    off[i] = selectLightOffset(xi[i], cdf, count, total);
    pdf[i] = off[i] < count ? lightPdfFromCdf(off[i], cdf, total) : 0.0f;
  }
}

// sampleLightPoint (:582-643) on primitive records (7 float4 each) with the two uniforms u[2 i],
// u[2 i + 1]; per case 7 floats (position, normal, area) and ok.
void ref_sample_light_point(const float *prims, const float *uv, uint32_t n, float *out, uint8_t *ok) {
  const float4 *P = reinterpret_cast<const float4 *>(prims);
  for (uint32_t i = 0; i < n; ++i) {
    set_tape(uv + 2ull * i, 2);
    uint32_t seed = 0;
    float3 p(0.0f), nn(0.0f);
    float area = 0.0f;
    const float4 *g = P + 7ull * i;
    ok[i] = sampleLightPoint(int(g[0].w), g[0], g[1], g[2], seed, p, nn, area) ? 1 : 0;
    const float vals[7] = {p.x, p.y, p.z, nn.x, nn.y, nn.z, area};
    std::memcpy(out + 7ull * i, vals, sizeof(vals));
  }
}

// scatter (Scatter.h:73-152) of a ray with direction dn[6 i..] hitting a surface with normal
// dn[6 i + 3..] (front[i]: front face) and decodeMaterial(material i, lod 1), drawing from the
// 4 uniforms tape4[4 i..]; per case the new direction, the weight and the draws used.
void ref_scatter(const float *dn, const uint8_t *front, const float *mats, const float *tape4, uint32_t n,
                 float *out_dir, float *out_w, uint32_t *draws) {
  const float4 *M = reinterpret_cast<const float4 *>(mats);
  for (uint32_t i = 0; i < n; ++i) {
    MaterialPayload m = decodeMaterial(int(i * kMaterialFloat4Count), M, 1.0f);
    set_tape(tape4 + 4ull * i, 4);
    Ray r;
    r.origin = float3(0.0f);
    r.direction = f3(dn + 6ull * i);
    intersection h;
    h.normal = f3(dn + 6ull * i + 3);
    h.frontFace = front[i] != 0;
    uint32_t seed = 0;
    float3 w = scatter(r, h, m, seed);
    out_dir[3 * i] = r.direction.x, out_dir[3 * i + 1] = r.direction.y, out_dir[3 * i + 2] = r.direction.z;
    out_w[3 * i] = w.x, out_w[3 * i + 1] = w.y, out_w[3 * i + 2] = w.z;
    draws[i] = seed;
  }
}

// A chain of restirUpdateReservoir calls (:97-115) with restirContribution / restirTarget-
// FromCandidate (:87-96) weights. Per chain k updates; update j of chain c reads cand[(c k + j)
// 16 floats] = light position xyz, light id, light normal xyz, area, pdf, radiance xyz,
// geometry factor, weight scale, sample count increment, unused, and draws its acceptance number
// from xi[c k + j]. The weight is (pdf > 0 ? target / pdf : 0) * weight scale. Per chain 18 floats:
// light position xyz, id, normal xyz, area, pdf, weight sum, sample count, selected weight,
// selected contribution xyz, valid, draws used, unused.
void ref_reservoir_chain(const float *cand, const float *xi, uint32_t chains, uint32_t k, float *out) {
  for (uint32_t c = 0; c < chains; ++c) {
    RestirReservoir r;
    set_tape(xi + (uint64_t)c * k, k);
    uint32_t seed = 0;
    for (uint32_t j = 0; j < k; ++j) {
      const float *q = cand + 16ull * ((uint64_t)c * k + j);
      LightSampleCandidate s;
      s.lightPosition = f3(q);
      s.lightId = (uint)q[3];
      s.lightNormal = f3(q + 4);
      s.lightArea = q[7];
      s.pdf = q[8];
      s.radiance = f3(q + 9);
      s.geometryFactor = q[12];
      float3 contribution = restirContribution(s);
      float target = restirTargetFromCandidate(s);
      float weight = (s.pdf > 0.0f ? target / s.pdf : 0.0f) * q[13];
      restirUpdateReservoir(r, s, contribution, weight, q[14], seed);
    }
    float *o = out + 18ull * c;
    const float vals[18] = {r.sample.lightPosition.x, r.sample.lightPosition.y, r.sample.lightPosition.z,
                            (float)r.sample.lightId, r.sample.lightNormal.x, r.sample.lightNormal.y,
                            r.sample.lightNormal.z, r.sample.lightArea, r.sample.pdf, r.weightSum, r.sampleCount,
                            r.selectedWeight, r.selectedContribution.x, r.selectedContribution.y,
                            r.selectedContribution.z, r.valid ? 1.0f : 0.0f, (float)seed, 0.0f};
    std::memcpy(o, vals, sizeof(vals));
  }
}

}  // extern "C"
