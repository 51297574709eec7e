// ORACLE — test infrastructure only (the checker of the wavefront path tracer).
//
// Scalar restatement of the reference's per-pixel path tracer:
//   pathTraceKernel raygen and averaging   Renderer/Shaders/PathTraceKernel.metal:67-162
//   rayColor bounce loop                   Renderer/Shaders/PathTracing.h:1168-1881
//     sky on miss :1211-1213, emission :1312-1317, one-sample NEE :1744-1848,
//     scatter + offset :1851-1861, Russian roulette :1863-1870, clamp :1879
//   decodeMaterial :165-196, evaluateDirectLightingBsdf :249-293, sampleLightPoint :582-643,
//   selectLightOffset :219-235, scatter / sampleCosineHemisphere / mirrorAngle Scatter.h:31-152
//   light CDF over active emissive primitives Renderer/Renderer.cpp:5161-5211, primitiveArea :1462-1480
// Contract changes (shared with the CUDA path tracer):
//   * random numbers: Philox4x32-10 (Salmon et al., SC'11) with key (seed_lo, seed_hi + frame)
//     and counter (pixel, sample, 4*bounce + block, view) instead of the reference's hash of the
//     pixel uv; block 0 = (light choice, light u1, light u2, lobe choice), block 1 = (direction
//     u1, direction u2, roulette, Fresnel choice), raygen = bounce 255 block 0;
//   * sin/cos(2 pi u), log2, exp2 and x^5 are defined by fixed polynomials/products (below) so
//     that host and device round identically;
//   * traversal and shadow visibility follow the contract (contract_core.h): lowest-index tie
//     rule, true any-hit shadow rays over (1e-4, dist - 0.001) for one-sample NEE (the reference's
//     acceptance window, PathTracing.h:1832-1834) and (1e-4, dist - 1e-4) for ReSTIR's
//     isLightVisible (:549-552);
//   * a path whose throughput becomes exactly zero stops (the reference keeps tracing it with no
//     effect on radiance);
//   * clamping to [0, 1] is optional (NOMAD_VIEW_CLAMP) so HDR radiance can be compared.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "contract_core.h"
#include "view_projection.h"

using namespace oracle_core;

namespace {

struct View {
  float cam[3], vu[3], vv[3], fp[3];
  uint32_t w, h, spp, maxDepth, seedLo, seedHi, frame, flags;
};
const uint32_t VIEW_CLAMP = 1u;
const float PI_F = 3.14159265358979323846f;

struct V {
  float x, y, z;
};
inline V v(float x, float y, float z) { return V{x, y, z}; }
inline V add(V a, V b) { return v(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V vsub(V a, V b) { return v(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V mul(V a, V b) { return v(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V scl(V a, float s) { return v(a.x * s, a.y * s, a.z * s); }
inline V dvs(V a, float s) { return v(a.x / s, a.y / s, a.z / s); }
inline V neg(V a) { return v(-a.x, -a.y, -a.z); }
inline float dt(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V crs(V a, V b) { return v(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline V nrmz(V a) {
  float l = std::sqrt(dt(a, a));
  return dvs(a, l);
}
inline bool fin(V a) { return std::isfinite(a.x) && std::isfinite(a.y) && std::isfinite(a.z); }
inline float mx(float a, float b) { return a < b ? b : a; }
inline float mn(float a, float b) { return b < a ? b : a; }
inline float c01(float x) { return mn(mx(x, 0.0f), 1.0f); }
inline V max0(V a) { return v(mx(a.x, 0.0f), mx(a.y, 0.0f), mx(a.z, 0.0f)); }
inline float lum(V c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }
inline V refl(V i, V n) { return vsub(i, scl(n, 2.0f * dt(n, i))); }
inline float p5(float x) {
  float x2 = x * x;
  return x2 * x2 * x;
}

// Philox4x32-10 from the paper: per round (hi0,lo0) = M0*c0, (hi1,lo1) = M1*c2,
// c = (hi1^c1^k0, lo1, hi0^c3^k1, lo0); keys bumped by the Weyl constants.
struct U4 {
  uint32_t x, y, z, w;
};
U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
    c = U4{(uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1, (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0};
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}
inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// Where a path's random numbers come from. Philox mode (tape == nullptr; the CUDA kernels'
// scheme): every draw has a fixed slot, a lane of a Philox block, and take() returns that slot's
// value, so a draw that a branch skips leaves every other draw unchanged. Tape mode: take()
// returns the caller's numbers in the order the draws are made and skip() drops one, which is the
// reference's scheme (u = randomFloat(seed); seed = random(seed), Random.h:6-17), where a skipped
// draw shifts the later ones. Every draw below is made at the point, and under the conditions,
// where the reference makes it, so the same code runs on identical numbers as the reference's
// shader code does when that code is handed the same tape (oracle/ref/ref_shade.cpp).
struct Draws {
  const float *tape = nullptr;
  uint32_t pos = 0, len = 0;
  float take(float slot) {
    if (!tape) return slot;
    const float u = pos < len ? tape[pos] : 0.5f;
    ++pos;
    return u;
  }
  void skip() {
    if (tape) ++pos;
  }
};

void sincos_turns(float u, float &s, float &c) {
  float t = u * 8.0f;
  float fo = std::floor(t);
  int o = (int)fo & 7;
  float x = (t - fo - 0.5f) * 0.785398163397448f;
  float x2 = x * x;
  float sx = x * (1.0f - x2 * (0.16666666666666667f - x2 * (0.008333333333333333f - x2 * 0.0001984126984126984f)));
  float cx = 1.0f - x2 * (0.5f - x2 * (0.041666666666666667f - x2 * (0.001388888888888889f - x2 * 2.48015873015873e-05f)));
  static const float kc[8] = {0.923879532511287f, 0.382683432365090f, -0.382683432365090f, -0.923879532511287f,
                              -0.923879532511287f, -0.382683432365090f, 0.382683432365090f, 0.923879532511287f};
  static const float ks[8] = {0.382683432365090f, 0.923879532511287f, 0.923879532511287f, 0.382683432365090f,
                              -0.382683432365090f, -0.923879532511287f, -0.923879532511287f, -0.382683432365090f};
  c = kc[o] * cx - ks[o] * sx;
  s = ks[o] * cx + kc[o] * sx;
}
float log2_series(float a) {
  int e;
  float m = std::frexp(a, &e);
  if (m < 0.70710678118654752f) {
    m = m * 2.0f;
    e -= 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float ln = 2.0f * s * (1.0f + s2 * (0.3333333333333333f + s2 * (0.2f + s2 * (0.14285714285714285f + s2 * 0.1111111111111111f))));
  return (float)e + ln * 1.4426950408889634f;
}
float exp2_series(float y) {
  if (y < -126.0f) return 0.0f;
  if (y > 127.0f) return INFINITY;
  float fi = std::floor(y);
  float f = (y - fi) * 0.6931471805599453f;
  float p = 1.0f + f * (1.0f + f * (0.5f + f * (0.16666666666666667f + f * (0.041666666666666667f +
            f * (0.008333333333333333f + f * (0.001388888888888889f + f * (0.0001984126984126984f +
            f * 2.48015873015873e-05f)))))));
  return std::ldexp(p, (int)fi);
}
float pow_pos(float a, float b) {
  if (!(a > 0.0f)) return 0.0f;
  return exp2_series(b * log2_series(a));
}

struct Mat {
  V diffuse;
  float opacity;
  V specular;
  float shininess;
  V emission;
  float power;
  V transmission;
  float ior, roughness;
};

Mat decode(const float *mats, int32_t prim, float lod) {
  const float *m = mats + 20ll * prim;
  Mat o;
  o.diffuse = max0(scl(v(m[0], m[1], m[2]), lod));
  o.opacity = c01(m[3]);
  o.specular = max0(v(m[4], m[5], m[6]));
  o.shininess = mx(m[7], 1.0f);
  o.emission = max0(v(m[8], m[9], m[10]));
  o.power = mx(m[11], 0.0f);
  o.transmission = max0(v(m[12], m[13], m[14]));
  o.ior = mx(m[15], 1e-3f);
  o.roughness = c01(m[19]);
  if (o.opacity < 1.0f && lum(o.transmission) <= 0.0f) {
    float t = 1.0f - o.opacity;
    o.transmission = v(t, t, t);
  }
  return o;
}

V geom_normal(const float *prims, int32_t prim, V p) {
  const float *g = prims + 28ll * prim;
  int type = (int)g[3];
  V sn = v(g[24], g[25], g[26]);
  if (type == 1) {
    V v0 = v(g[0], g[1], g[2]);
    V fb = crs(vsub(v(g[4], g[5], g[6]), v0), vsub(v(g[8], g[9], g[10]), v0));
    fb = dt(fb, fb) > 0.0f ? nrmz(fb) : v(0.0f, 1.0f, 0.0f);
    V n = (dt(sn, sn) > RAY_EPS && fin(sn)) ? nrmz(sn) : fb;
    if (!fin(n) || dt(n, n) <= RAY_EPS) n = fb;
    return n;
  }
  if (type == 2) {
    V fb = crs(v(g[4], g[5], g[6]), v(g[8], g[9], g[10]));
    fb = (dt(fb, fb) > RAY_EPS && fin(fb)) ? nrmz(fb) : v(0.0f, 1.0f, 0.0f);
    return (dt(sn, sn) > RAY_EPS && fin(sn)) ? nrmz(sn) : fb;
  }
  return nrmz(vsub(p, v(g[0], g[1], g[2])));
}

V bsdf(const Mat &m, V normal, V viewDir, V lightDir) {
  V n = nrmz(normal), vv = nrmz(viewDir), l = nrmz(lightDir);
  if (!fin(n) || !fin(vv) || !fin(l)) return v(0, 0, 0);
  float nl = mx(dt(n, l), 0.0f), nv = mx(dt(n, vv), 0.0f);
  if (nl <= 0.0f || nv <= 0.0f) return v(0, 0, 0);
  V dc = scl(max0(m.diffuse), m.opacity);
  V sc0 = scl(m.specular, m.opacity);
  V sc = v(c01(sc0.x), c01(sc0.y), c01(sc0.z));
  float rough = c01(m.roughness);
  float alpha = mx(rough * rough, 0.001f);
  float a2 = alpha * alpha;
  V h = nrmz(add(vv, l));
  float nh = mx(dt(n, h), 0.0f), vh = mx(dt(vv, h), 0.0f);
  float den = nh * nh * (a2 - 1.0f) + 1.0f;
  float D = a2 / mx(PI_F * den * den, RAY_EPS);
  float k = alpha + 1.0f;
  k = (k * k) / 8.0f;
  float G = (nv / (nv * (1.0f - k) + k)) * (nl / (nl * (1.0f - k) + k));
  float Fc = p5(mx(1.0f - vh, 0.0f));
  V F = add(sc, scl(vsub(v(1, 1, 1), sc), Fc));
  V spec = dvs(scl(F, D * G), mx(4.0f * nl * nv, RAY_EPS));
  return add(dvs(dc, PI_F), spec);
}

void onb(V n, V &t, V &b) {
  V up = std::fabs(n.z) < 0.999f ? v(0, 0, 1) : v(0, 1, 0);
  t = nrmz(crs(up, n));
  b = nrmz(crs(n, t));
}

V scatter(V inDir, V normal, bool front, const Mat &m, Draws &dr, float xiLobe, float u1, float u2, float xiF,
          V &out) {
  float dw = mx(lum(m.diffuse) * m.opacity, 0.0f);
  float sw = mx(lum(m.specular) * m.opacity, 0.0f);
  float tw = mx(lum(m.transmission) * (1.0f - m.opacity), 0.0f);
  if (tw > 0.0f) sw = 0.0f;
  float total = dw + sw + tw;
  if (total <= 0.0f) {
    out = normal;
    return v(0, 0, 0);
  }
  float xi = dr.take(xiLobe) * total;
  if (xi < dw) {
    u1 = dr.take(u1);
    u2 = dr.take(u2);
    float r = std::sqrt(mx(0.0f, u1));
    float s, c;
    sincos_turns(u2, s, c);
    float x = r * c, y = r * s, z = std::sqrt(mx(0.0f, 1.0f - u1));
    V t, b;
    onb(normal, t, b);
    out = nrmz(add(add(scl(t, x), scl(b, y)), scl(normal, z)));
    return dvs(scl(m.diffuse, m.opacity), mx(dw / total, 1e-4f));
  }
  xi = xi - dw;
  if (xi < sw) {
    V rd = refl(inDir, normal);
    float ex = mx(m.shininess, 1.0f);
    if (m.roughness > 0.0f) {
      float sm = c01(1.0f - m.roughness);
      ex = mx(ex, mx(1.0f, sm * sm * 256.0f));
    }
    u1 = dr.take(u1);
    u2 = dr.take(u2);
    float ct = pow_pos(u1, 1.0f / (ex + 1.0f));
    float st = std::sqrt(mx(0.0f, 1.0f - ct * ct));
    float s, c;
    sincos_turns(u2, s, c);
    V t, b;
    onb(rd, t, b);
    out = nrmz(add(add(scl(t, st * c), scl(b, st * s)), scl(rd, ct)));
    return dvs(m.specular, mx(sw / total, 1e-4f));
  }
  float prob = mx(tw / total, 1e-4f);
  float eta = mx(m.ior, 1e-3f);
  float ratio = front ? (1.0f / eta) : eta;
  float cosT = dt(neg(inDir), normal);
  float sinT = std::sqrt(mx(0.0f, 1.0f - cosT * cosT));
  float r0 = (1.0f - ratio) / (1.0f + ratio);
  r0 = r0 * r0;
  float refl_ = r0 + (1.0f - r0) * p5(1.0f - cosT);
  xiF = dr.take(xiF);
  if ((ratio * sinT > 1.0f) || (refl_ > xiF)) {
    out = refl(inDir, normal);
    return dvs(m.specular, prob);
  }
  float d = dt(normal, inDir);
  float k = 1.0f - ratio * ratio * (1.0f - d * d);
  if (k < 0.0f) {
    out = refl(inDir, normal);
    return dvs(m.specular, prob);
  }
  V rr = vsub(scl(inDir, ratio), scl(normal, ratio * d + std::sqrt(k)));
  if (!fin(rr)) {
    out = refl(inDir, normal);
    return dvs(m.specular, prob);
  }
  out = nrmz(rr);
  return dvs(m.transmission, prob);
}

bool light_point(const float *prims, uint32_t lp, Draws &dr, float u1, float u2, V &pos, V &nrm, float &area) {
  const float *g = prims + 28ll * lp;
  int type = (int)g[3];
  if (type == 0) {
    float radius = g[4];
    if (radius <= 0.0f) return false;
    u1 = dr.take(u1);
    u2 = dr.take(u2);
    float z = 2.0f * u1 - 1.0f;
    float s, c;
    sincos_turns(u2, s, c);
    float r = std::sqrt(mx(0.0f, 1.0f - z * z));
    V dir = v(r * c, r * s, z);
    pos = add(v(g[0], g[1], g[2]), scl(dir, radius));
    nrm = dir;
    area = 4.0f * PI_F * radius * radius;
    return area > 0.0f;
  }
  if (type == 1) {
    u1 = dr.take(u1);
    u2 = dr.take(u2);
    float su1 = std::sqrt(u1);
    float b0 = 1.0f - su1, b1 = su1 * (1.0f - u2), b2 = su1 * u2;
    V v0 = v(g[0], g[1], g[2]), v1 = v(g[4], g[5], g[6]), v2 = v(g[8], g[9], g[10]);
    pos = add(add(scl(v0, b0), scl(v1, b1)), scl(v2, b2));
    V n = crs(vsub(v1, v0), vsub(v2, v0));
    float ln = std::sqrt(dt(n, n));
    if (ln <= 0.0f) return false;
    nrm = dvs(n, ln);
    area = 0.5f * ln;
    return area > 0.0f;
  }
  if (type == 2) {
    u1 = dr.take(u1);
    u2 = dr.take(u2);
    float su = u1 * 2.0f - 1.0f, sv = u2 * 2.0f - 1.0f;
    V c = v(g[0], g[1], g[2]), e1 = v(g[4], g[5], g[6]), e2 = v(g[8], g[9], g[10]);
    pos = add(add(c, scl(e1, su)), scl(e2, sv));
    V n = crs(e1, e2);
    float ln = std::sqrt(dt(n, n));
    if (ln <= 0.0f) return false;
    nrm = dvs(n, ln);
    area = 4.0f * ln;
    return area > 0.0f;
  }
  return false;
}

struct LightsH {
  std::vector<uint32_t> idx;
  std::vector<float> cdf;
  float total = 0.0f;
};

LightsH build_lights(const float *prims, const float *mats, const uint8_t *active, const int32_t *blasRoot,
                     const int32_t *primObject, uint32_t primCount) {
  LightsH L;
  float total = 0.0f;
  for (uint32_t i = 0; i < primCount; ++i) {
    if (!active[i] || blasRoot[primObject[i]] < 0) continue;
    const float *m = mats + 20ull * i;
    float strength = m[11] * (m[8] * 0.2126f + m[9] * 0.7152f + m[10] * 0.0722f);
    if (!(strength > 0.0f)) continue;
    const float *g = prims + 28ull * i;
    int type = (int)g[3];
    float area;
    if (type == 0) {
      area = 4.0f * PI_F * g[4] * g[4];
    } else {
      V a = type == 1 ? vsub(v(g[4], g[5], g[6]), v(g[0], g[1], g[2])) : v(g[4], g[5], g[6]);
      V b = type == 1 ? vsub(v(g[8], g[9], g[10]), v(g[0], g[1], g[2])) : v(g[8], g[9], g[10]);
      V c = crs(a, b);
      float len = std::sqrt(c.x * c.x + c.y * c.y + c.z * c.z);
      area = type == 1 ? 0.5f * len : 4.0f * len;
    }
    if (!(area > 0.0f)) continue;
    float w = area * strength;
    if (!(w > 0.0f)) continue;
    total += w;
    L.idx.push_back(i);
    L.cdf.push_back(total);
  }
  L.total = total;
  return L;
}

uint32_t select_light(float xi, const LightsH &L) {
  uint32_t n = (uint32_t)L.idx.size();
  float target = xi * L.total;
  uint32_t lo = 0, hi = n;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (L.cdf[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  return lo < n - 1 ? lo : n - 1;
}

// lightPdfFromCdf (PathTracing.h:237-247): the chosen slot's share of the total weight.
float light_pdf(const LightsH &L, uint32_t off) {
  float prev = off > 0 ? L.cdf[off - 1] : 0.0f;
  float w = L.cdf[off] - prev;
  return (L.total > 0.0f && w > 0.0f) ? w / L.total : 0.0f;
}

// The per-primitive light pdf the reservoir reuse reads (lightPdfLookup, Renderer.cpp:5195-5208).
std::vector<float> light_pdf_lookup(const LightsH &L, uint32_t prim_count) {
  std::vector<float> out(prim_count, 0.0f);
  for (size_t k = 0; k < L.idx.size(); ++k) {
    float w = L.cdf[k] - (k ? L.cdf[k - 1] : 0.0f);
    if (w > 0.0f && L.total > 0.0f) out[L.idx[k]] = w / L.total;
  }
  return out;
}

struct Ctx {
  Scene s;
  const float *mats;
  LightsH L;
  uint32_t objectCount;
};

Ray mkray(V o, V d, float tmax) { return Ray{mk(o.x, o.y, o.z), mk(d.x, d.y, d.z), tmax}; }

Hit closest(const Ctx &c, const Ray &r) {
  Hit h{r.tmax, 0.0f, 0.0f, -1, -1};
  trace_near_first<false>(c.s, r, h, nullptr);
  if (h.prim < 0) h.t = INFINITY;
  return h;
}
// Reference rules for the shading pin (oracle_set_reference_rules; off by default, and off for
// everything the CUDA path is checked against):
//   kRuleVisibility: light visibility by the reference's own test, a closest hit over the whole
//     ray, visible iff nothing is hit or the hit is the light primitive itself at t >= dist - eps
//     (isLightVisible :549-552, NEE :1828-1834), instead of the contract's any-hit over
//     (1e-4, dist - eps). They differ only when the light is numerically missed with something
//     behind it, or an occluder lies within eps in front of the light; the counters record how
//     many shadow decisions the two rules take differently.
//   kRuleReprojection: ReSTIR reference mode finds the temporal source pixel through the float
//     view-projection matrix the pin hands the reference, with the reference's arithmetic
//     (view_projection.h), instead of the contract's ray-plane intersection with the previous
//     view; the two round differently within a hair of a pixel boundary.
constexpr int kRuleVisibility = 1, kRuleReprojection = 2;
std::atomic<int> g_vis_rule{0}, g_vis_track{0};
std::atomic<uint64_t> g_vis_tests{0}, g_vis_differ{0};

bool occluded(const Ctx &c, const Ray &r);

// Is the light primitive `lp`, sampled at distance dist, visible along r (r.tmax = dist - eps,
// at least 1e-4)? Counts rule disagreements while tracking is on.
bool light_visible(const Ctx &c, const Ray &r, int32_t lp, float dist, float eps) {
  const bool contractVis = !occluded(c, r);
  if (!(g_vis_rule.load(std::memory_order_relaxed) & kRuleVisibility) && !g_vis_track.load(std::memory_order_relaxed))
    return contractVis;
  Hit h{INFINITY, 0.0f, 0.0f, -1, -1};
  Ray full = r;
  full.tmax = INFINITY;
  trace_near_first<false>(c.s, full, h, nullptr);
  const bool refVis = h.prim < 0 || (h.prim == lp && h.t >= dist - eps);
  g_vis_tests.fetch_add(1, std::memory_order_relaxed);
  if (refVis != contractVis) g_vis_differ.fetch_add(1, std::memory_order_relaxed);
  return (g_vis_rule.load(std::memory_order_relaxed) & kRuleVisibility) ? refVis : contractVis;
}

bool occluded(const Ctx &c, const Ray &r) {
  Hit h{r.tmax, 0.0f, 0.0f, -1, -1};
  trace_near_first<true>(c.s, r, h, nullptr);
  return h.prim >= 0;
}

// One path; returns its radiance (unclamped) and counts closest hits per object.
// Precomputed ReSTIR result of one path: the shadow ray and its unoccluded contribution.
struct RestirOut {
  bool valid = false;
  bool direct = false;  // reference mode: visibility already applied, added as is
  V origin, dir, contrib;
  float tmax = 0.0f;
  uint32_t tapePos = 0;  // tape mode: where the rest of the path continues drawing
};
const uint32_t VIEW_RESTIR = 2u;

// Tape mode: the pixel's two jitter numbers are drawn first, as pathTraceKernel draws them
// (PathTraceKernel.metal:91-94), whether or not the view jitters.
V path(const Ctx &c, const View &vw, uint32_t vi, uint32_t pixel, uint32_t sample, uint32_t *objHits,
       uint64_t *stats, const RestirOut *rs, Draws &dr) {
  uint32_t k0 = vw.seedLo, k1 = vw.seedHi + vw.frame;
  uint32_t px = pixel % vw.w, py = pixel / vw.w;
  U4 r0 = philox(U4{pixel, sample, 255u * 4u, vi}, k0, k1);
  float ux = ((float)px + 0.5f) / (float)vw.w, uy = ((float)py + 0.5f) / (float)vw.h;
  bool center = (vw.flags & 4u) != 0;
  const float jx = dr.take(u01(r0.x)), jy = dr.take(u01(r0.y));
  if (dr.tape && rs) dr.pos = rs->tapePos;  // the ReSTIR pass drew the pixel's numbers up to here
  float s = ux + (center ? 0.0f : (jx - 0.5f) / (float)vw.w);
  float t = uy + (center ? 0.0f : (jy - 0.5f) / (float)vw.h);
  V d = v(vw.fp[0] + s * vw.vu[0] + t * vw.vv[0] - vw.cam[0], vw.fp[1] + s * vw.vu[1] + t * vw.vv[1] - vw.cam[1],
          vw.fp[2] + s * vw.vu[2] + t * vw.vv[2] - vw.cam[2]);
  V dir = nrmz(d);
  V org = v(vw.cam[0], vw.cam[1], vw.cam[2]);
  float dx[3] = {vw.vu[0] / (float)vw.w, vw.vu[1] / (float)vw.w, vw.vu[2] / (float)vw.w};
  float dy[3] = {vw.vv[0] / (float)vw.h, vw.vv[1] / (float)vw.h, vw.vv[2] / (float)vw.h};
  float cx = dx[1] * dy[2] - dx[2] * dy[1], cy = dx[2] * dy[0] - dx[0] * dy[2], cz = dx[0] * dy[1] - dx[1] * dy[0];
  float lod = 1.0f / (1.0f + std::sqrt(cx * cx + cy * cy + cz * cz));
  V thr = v(1, 1, 1), rad = v(0, 0, 0);
  for (uint32_t depth = 0; depth < vw.maxDepth; ++depth) {
    stats[0]++;
    Ray ray = mkray(org, dir, INFINITY);
    Hit h = closest(c, ray);
    if (h.prim < 0) {
      stats[1]++;
      V ud = nrmz(dir);
      float sk = 0.5f * (ud.y + 1.0f);
      V sky = v(1.0f + (0.6f - 1.0f) * sk, 1.0f + (0.7f - 1.0f) * sk, 1.0f + (1.0f - 1.0f) * sk);
      rad = add(rad, mul(thr, sky));
      break;
    }
    stats[3]++;
    if (objHits) objHits[h.inst]++;
    U4 b0 = philox(U4{pixel, sample, depth * 4u + 0u, vi}, k0, k1);
    U4 b1 = philox(U4{pixel, sample, depth * 4u + 1u, vi}, k0, k1);
    V p = v(org.x + h.t * dir.x, org.y + h.t * dir.y, org.z + h.t * dir.z);
    V n = geom_normal(c.s.prims, h.prim, p);
    bool front = dt(n, dir) < 0.0f;
    if (!front) n = neg(n);
    Mat m = decode(c.mats, h.prim, lod);
    if (m.power * lum(m.emission) > 0.0f) rad = add(rad, scl(mul(thr, m.emission), m.power));
    V dc = scl(m.diffuse, m.opacity);
    bool restirHere = depth == 0 && (vw.flags & VIEW_RESTIR) != 0;
    if (restirHere) {
      if (rs && rs->valid) {
        stats[2]++;
        if (rs->direct || !occluded(c, mkray(rs->origin, rs->dir, rs->tmax))) rad = add(rad, rs->contrib);
      }
    } else if (lum(dc) > 0.0f && !c.L.idx.empty() && c.L.total > 0.0f) {
      uint32_t off = select_light(dr.take(u01(b0.x)), c.L);
      uint32_t lp = c.L.idx[off];
      V lpos, lnrm;
      float area = 0.0f;
      if ((int32_t)lp != h.prim && light_point(c.s.prims, lp, dr, u01(b0.y), u01(b0.z), lpos, lnrm, area) &&
          area > 0.0f) {
        V toL = vsub(lpos, p);
        float d2 = dt(toL, toL);
        if (d2 > RAY_EPS) {
          float dist = std::sqrt(d2);
          V wi = dvs(toL, dist);
          float cosT = mx(dt(n, wi), 0.0f), cosL = mx(dt(lnrm, neg(wi)), 0.0f);
          if (cosT > 0.0f && cosL > 0.0f) {
            float lpdf = light_pdf(c.L, off);
            if (lpdf > 0.0f) {
              float totalPdf = lpdf * ((1.0f / area) * d2 / cosL);
              if (totalPdf > 0.0f) {
                // visible when the closest hit is the light itself at t >= dist - 0.001
                // (PathTracing.h:1832-1834): the any-hit window ends there
                float tmax = dist - 0.001f;
                if (tmax < RAY_EPS) tmax = RAY_EPS;
                stats[2]++;
                Ray sr = mkray(add(p, scl(n, 0.0005f)), wi, tmax);
                if (light_visible(c, sr, (int32_t)lp, dist, 0.001f)) {
                  Mat lm = decode(c.mats, (int32_t)lp, 1.0f);
                  V lrad = scl(lm.emission, lm.power);
                  V b = bsdf(m, n, nrmz(neg(dir)), wi);
                  rad = add(rad, scl(mul(mul(thr, b), lrad), cosT / totalPdf));
                }
              }
            }
          }
        }
      }
    }
    V nd;
    V wgt = scatter(dir, n, front, m, dr, u01(b0.w), u01(b1.x), u01(b1.y), u01(b1.w), nd);
    dr.skip();  // the reference advances its seed once more after scatter (PathTracing.h:1855)
    V bias = dt(nd, n) < 0.0f ? neg(n) : n;
    org = add(p, scl(bias, RAY_EPS));
    dir = nd;
    thr = mul(thr, wgt);
    if (depth >= 5) {
      float pm = mx(thr.x, mx(thr.y, thr.z));
      if (dr.take(u01(b1.z)) >= pm) break;
      thr = dvs(thr, pm);
    }
    if (thr.x == 0.0f && thr.y == 0.0f && thr.z == 0.0f) break;
  }
  return rad;
}

int render_impl(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                const float *materials, const int32_t *prim_indices, const uint8_t *active,
                const int32_t *blas_root, const int32_t *prim_object, uint32_t object_count,
                uint32_t prim_count, const void *views, uint32_t nviews, const uint64_t *pixels,
                uint64_t npix, float *out, uint32_t *obj_hits, uint64_t *stats, uint32_t threads,
                const float *tapes, uint32_t tape_len) {
  if (!bvh || !tlas || !prims || !materials || !views || !out || !pixels) return 1;
  Ctx c{{bvh, tlas, tlas_count, prims, prim_indices, active, blas_root, prim_object}, materials, {}, object_count};
  c.L = build_lights(prims, materials, active, blas_root, prim_object, prim_count);
  const View *vs = static_cast<const View *>(views);
  std::vector<uint64_t> voff(nviews + 1, 0);
  for (uint32_t i = 0; i < nviews; ++i) voff[i + 1] = voff[i] + (uint64_t)vs[i].w * vs[i].h;
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  std::vector<std::vector<uint32_t>> hits(threads, std::vector<uint32_t>(obj_hits ? object_count : 0, 0));
  std::vector<std::vector<uint64_t>> st(threads, std::vector<uint64_t>(4, 0));
  std::atomic<uint64_t> next{0};
  auto work = [&](uint32_t tid) {
    for (;;) {
      uint64_t b = next.fetch_add(64);
      if (b >= npix) break;
      uint64_t e = std::min<uint64_t>(npix, b + 64);
      for (uint64_t q = b; q < e; ++q) {
        uint64_t g = pixels[q];
        uint32_t vi = 0;
        while (vi + 1 < nviews && voff[vi + 1] <= g) ++vi;
        const View &vw = vs[vi];
        uint32_t pixel = (uint32_t)(g - voff[vi]);
        bool cl = (vw.flags & VIEW_CLAMP) != 0;
        float ax = 0.0f, ay = 0.0f, az = 0.0f;
        Draws dr;  // tape mode: one tape per listed pixel, drawn on across its samples
        if (tapes) dr = Draws{tapes + q * tape_len, 0, tape_len};
        for (uint32_t s = 0; s < vw.spp; ++s) {
          V r = path(c, vw, vi, pixel, s, obj_hits ? hits[tid].data() : nullptr, st[tid].data(), nullptr, dr);
          if (cl) r = v(c01(r.x), c01(r.y), c01(r.z));
          ax = ax + r.x;
          ay = ay + r.y;
          az = az + r.z;
        }
        float ns = (float)vw.spp;
        ax = ax / ns;
        ay = ay / ns;
        az = az / ns;
        if (cl) {
          ax = c01(ax);
          ay = c01(ay);
          az = c01(az);
        }
        out[3 * q] = ax;
        out[3 * q + 1] = ay;
        out[3 * q + 2] = az;
      }
    }
  };
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; ++t) pool.emplace_back(work, t);
  for (auto &t : pool) t.join();
  if (obj_hits)
    for (auto &hh : hits)
      for (uint32_t o = 0; o < object_count; ++o) obj_hits[o] += hh[o];
  if (stats)
    for (auto &s : st)
      for (int k = 0; k < 4; ++k) stats[k] += s[k];
  return 0;
}

}  // namespace

extern "C" {

// Renders the listed pixels (global pixel indices over the concatenated views) into out
// (3 floats per listed pixel). views: nomad_view structs. obj_hits (object_count counters) and
// stats (4 counters: rays, escapes, shadow rays, hits) may be null; they accumulate over the
// listed pixels only.
int oracle_render(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                  const float *materials, const int32_t *prim_indices, const uint8_t *active,
                  const int32_t *blas_root, const int32_t *prim_object, uint32_t object_count,
                  uint32_t prim_count, const void *views, uint32_t nviews, const uint64_t *pixels,
                  uint64_t npix, float *out, uint32_t *obj_hits, uint64_t *stats, uint32_t threads) {
  return render_impl(bvh, tlas, tlas_count, prims, materials, prim_indices, active, blas_root, prim_object,
                     object_count, prim_count, views, nviews, pixels, npix, out, obj_hits, stats, threads,
                     nullptr, 0);
}

// oracle_render in tape mode: `tapes` holds tape_len uniforms per listed pixel, drawn in the
// reference's order (Draws), so the output can be compared with the reference's own
// pathTraceKernel / rayColor run on the same numbers.
int oracle_render_tape(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                       const float *materials, const int32_t *prim_indices, const uint8_t *active,
                       const int32_t *blas_root, const int32_t *prim_object, uint32_t object_count,
                       uint32_t prim_count, const void *views, uint32_t nviews, const uint64_t *pixels,
                       uint64_t npix, float *out, uint32_t threads, const float *tapes, uint32_t tape_len) {
  if (!tapes || tape_len == 0) return 1;
  return render_impl(bvh, tlas, tlas_count, prims, materials, prim_indices, active, blas_root, prim_object,
                     object_count, prim_count, views, nviews, pixels, npix, out, nullptr, nullptr, threads,
                     tapes, tape_len);
}

}  // extern "C"

extern "C" void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  U4 r = philox(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
  out[3] = r.w;
}

extern "C" void oracle_math(float u, float out[4]) {
  sincos_turns(u, out[0], out[1]);
  out[2] = log2_series(u > 0.0f ? u : 1.0f);
  out[3] = exp2_series(-u * 4.0f);
}

// ---------------------------------------------------------------------------------------------
// ReSTIR DI (config mode), restated pass by pass in the CUDA core's order: initial RIS for all
// paths, temporal reuse for all paths, spatial reuse for all paths, final sample + shadow ray,
// then the rest of every path. Reservoirs and surfaces use the device layout
// (12 floats each) so consecutive frames can be chained through the caller.
namespace {

struct ResvH {
  float a[4], b[4], c[4];
};
struct SurfH {
  float p[4], n[4], v[4];
};
inline int32_t fbi(float f) {
  int32_t i;
  std::memcpy(&i, &f, 4);
  return i;
}
inline float ibf(int32_t i) {
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}
ResvH resv_empty() {
  ResvH r{};
  r.a[3] = ibf(-1);
  return r;
}

float restir_target(const Ctx &c, const Mat &m, const SurfH &s, V lpos, V lnrm, int32_t lp, V &fa, V &wi,
                    float &dist) {
  fa = v(0, 0, 0);
  if (lp < 0 || lp == fbi(s.n[3])) return 0.0f;
  V p = v(s.p[0], s.p[1], s.p[2]), n = v(s.n[0], s.n[1], s.n[2]);
  V toL = vsub(lpos, p);
  float d2 = dt(toL, toL);
  if (d2 <= RAY_EPS) return 0.0f;
  dist = std::sqrt(d2);
  wi = dvs(toL, dist);
  float cosT = mx(dt(n, wi), 0.0f), cosL = mx(dt(lnrm, neg(wi)), 0.0f);
  if (cosT <= 0.0f || cosL <= 0.0f) return 0.0f;
  Mat lm = decode(c.mats, lp, 1.0f);
  V lrad = scl(lm.emission, lm.power);
  V f = scl(mul(bsdf(m, n, v(s.v[0], s.v[1], s.v[2]), wi), lrad), cosT);
  float g = cosL / mx(d2, RAY_EPS);
  fa = scl(f, g);
  return mx(lum(fa), 0.0f);
}

bool restir_gate(const SurfH &s, const SurfH &q) {
  if (q.v[3] <= 0.0f) return false;
  float depth = s.p[3];
  V dp = vsub(v(q.p[0], q.p[1], q.p[2]), v(s.p[0], s.p[1], s.p[2]));
  float posTh = mx(0.01f * depth, 0.02f), depTh = mx(0.02f * depth, 0.05f);
  if (!(std::sqrt(dt(dp, dp)) <= posTh)) return false;
  if (!(std::fabs(q.p[3] - depth) <= depTh)) return false;
  V qn = v(q.n[0], q.n[1], q.n[2]);
  if (!(dt(qn, qn) > RAY_EPS)) return false;
  return dt(nrmz(qn), nrmz(v(s.n[0], s.n[1], s.n[2]))) >= 0.9f;
}

void restir_merge(const Ctx &c, ResvH &out, const ResvH &src, const SurfH &s, const Mat &m, float capM, float u) {
  int32_t lp = fbi(src.a[3]);
  if (lp < 0 || !(src.c[2] > 0.0f) || !(src.c[1] > 0.0f) || !(src.c[3] > 0.0f)) return;
  float Mp = mn(src.c[2], capM);
  float Wp = src.c[1] / (src.c[2] * src.c[3]);
  V fa, wi;
  float dist;
  float ph = restir_target(c, m, s, v(src.a[0], src.a[1], src.a[2]), v(src.b[0], src.b[1], src.b[2]), lp, fa, wi, dist);
  float w = ph * Wp * Mp;
  out.c[1] = out.c[1] + w;
  out.c[2] = out.c[2] + Mp;
  if (w > 0.0f && u * out.c[1] < w) {
    std::memcpy(out.a, src.a, 16);
    std::memcpy(out.b, src.b, 16);
    out.c[3] = ph;
  }
}

// ---- reference mode (the reference's own ReSTIR, PathTracing.h:308-480, :1363-1742) ----
// Reservoir layout: a = (light position, bits(light primitive)), b = (light normal, 1 / area),
// c = (candidate pdf, weight sum, sample count, selected weight).
struct RefC {
  V lpos, lnrm, wi, radG;
  float invArea, dist, pdf;
  int32_t lp;
};

// Candidate geometry before the visibility test (sampleDirectLightCandidate :344-371,
// buildRestirCandidateFromStored :414-438).
bool ref_geometry(const SurfH &s, const Mat &m, V lpos, V lnrm, float invArea, float lightPdf, V lrad, int32_t lp,
                  RefC &c) {
  V p = v(s.p[0], s.p[1], s.p[2]), n = v(s.n[0], s.n[1], s.n[2]);
  V toL = vsub(lpos, p);
  float d2 = dt(toL, toL);
  if (d2 <= RAY_EPS) return false;
  float dist = std::sqrt(d2);
  V wi = dvs(toL, dist);
  float cosT = mx(dt(n, wi), 0.0f), cosL = mx(dt(lnrm, neg(wi)), 0.0f);
  if (cosT <= 0.0f || cosL <= 0.0f) return false;
  if (lightPdf <= 0.0f) return false;
  float pdfSolid = invArea * d2 / cosL;
  float pdf = lightPdf * pdfSolid;
  if (pdf <= 0.0f) return false;
  V rad = scl(mul(bsdf(m, n, v(s.v[0], s.v[1], s.v[2]), wi), lrad), cosT);
  float g = cosL / mx(d2, RAY_EPS);
  c = RefC{lpos, lnrm, wi, scl(rad, g), invArea, dist, pdf, lp};
  return true;
}

// isLightVisible (:503-556) as the contract's any-hit: origin offset 5e-4 along the normal.
bool ref_visible(const Ctx &cx, const SurfH &s, const RefC &c) {
  float tmax = c.dist - RAY_EPS;
  if (tmax < RAY_EPS) tmax = RAY_EPS;
  V o = add(v(s.p[0], s.p[1], s.p[2]), scl(v(s.n[0], s.n[1], s.n[2]), 5.0f * RAY_EPS));
  return light_visible(cx, mkray(o, c.wi, tmax), c.lp, c.dist, RAY_EPS);
}

// restirUpdateReservoir (:97-115): the acceptance number is drawn only for a positive weight.
void ref_update(ResvH &r, V &contrib, const RefC &c, V cc, float w, float inc, Draws &dr, float xiSlot) {
  if (w <= 0.0f || inc <= 0.0f) return;
  r.c[1] = r.c[1] + w;
  r.c[2] = r.c[2] + inc;
  const float xi = dr.take(xiSlot);
  if (fbi(r.a[3]) < 0 || xi * r.c[1] < w) {
    r.a[0] = c.lpos.x; r.a[1] = c.lpos.y; r.a[2] = c.lpos.z; r.a[3] = ibf(c.lp);
    r.b[0] = c.lnrm.x; r.b[1] = c.lnrm.y; r.b[2] = c.lnrm.z; r.b[3] = c.invArea;
    r.c[0] = c.pdf;
    r.c[3] = w;
    contrib = cc;
  }
}

float view_lod(const View &vw) {
  float dx[3] = {vw.vu[0] / (float)vw.w, vw.vu[1] / (float)vw.w, vw.vu[2] / (float)vw.w};
  float dy[3] = {vw.vv[0] / (float)vw.h, vw.vv[1] / (float)vw.h, vw.vv[2] / (float)vw.h};
  float cx = dx[1] * dy[2] - dx[2] * dy[1], cy = dx[2] * dy[0] - dx[0] * dy[2], cz = dx[0] * dy[1] - dx[1] * dy[0];
  return 1.0f / (1.0f + std::sqrt(cx * cx + cy * cy + cz * cz));
}

}  // namespace

namespace {

int restir_impl(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                const float *materials, const int32_t *prim_indices, const uint8_t *active,
                const int32_t *blas_root, const int32_t *prim_object, uint32_t object_count,
                uint32_t prim_count, const void *views, uint32_t nviews, const uint32_t *cfg_u,
                const float *cfg_f, const float *prev_resv, const float *prev_surf,
                const void *prev_views, int have_prev, float *out_resv, float *out_surf,
                float *out_rgb, uint64_t *stats, uint32_t threads, const float *tapes, uint32_t tape_len) {
  Ctx c{{bvh, tlas, tlas_count, prims, prim_indices, active, blas_root, prim_object}, materials, {}, object_count};
  c.L = build_lights(prims, materials, active, blas_root, prim_object, prim_count);
  const View *vs = static_cast<const View *>(views);
  const View *pvs = static_cast<const View *>(prev_views);
  const uint32_t C = cfg_u[0], temporal = cfg_u[1], spatialN = cfg_u[2];
  const float radius = cfg_f[0], capM = cfg_f[1] * (float)C;
  std::vector<uint64_t> poff(nviews + 1, 0), xoff(nviews + 1, 0);
  for (uint32_t i = 0; i < nviews; ++i) {
    poff[i + 1] = poff[i] + (uint64_t)vs[i].w * vs[i].h * vs[i].spp;
    xoff[i + 1] = xoff[i] + (uint64_t)vs[i].w * vs[i].h;
  }
  const uint64_t P = poff[nviews];
  auto view_of = [&](uint64_t pid) {
    uint32_t i = 0;
    while (i + 1 < nviews && poff[i + 1] <= pid) ++i;
    return i;
  };
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  auto par = [&](auto fn) {
    std::atomic<uint64_t> next{0};
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < threads; ++t)
      pool.emplace_back([&, t]() {
        for (;;) {
          uint64_t b = next.fetch_add(64);
          if (b >= P) break;
          for (uint64_t q = b; q < std::min<uint64_t>(P, b + 64); ++q) fn(q, t);
        }
      });
    for (auto &th : pool) th.join();
  };
  std::vector<ResvH> rInit(P), rTemp(P);
  ResvH *rFin = reinterpret_cast<ResvH *>(out_resv);
  SurfH *sCur = reinterpret_cast<SurfH *>(out_surf);
  const ResvH *rPrev = reinterpret_cast<const ResvH *>(prev_resv);
  const SurfH *sPrev = reinterpret_cast<const SurfH *>(prev_surf);
  const bool refMode = cfg_u[3] != 0;
  std::vector<RestirOut> roAll;
  std::vector<std::vector<uint64_t>> refStats(threads, std::vector<uint64_t>(4, 0));
  if (refMode) {
    const std::vector<float> lpdfOf = light_pdf_lookup(c.L, prim_count);
    roAll.resize(P);
    par([&](uint64_t pid, uint32_t tid) {
      uint32_t vi = view_of(pid);
      const View &vw = vs[vi];
      ResvH r = resv_empty();
      SurfH s{};
      V contrib = v(0, 0, 0);
      RestirOut ro;
      uint64_t local = pid - poff[vi];
      uint32_t pixel = (uint32_t)(local / vw.spp), sample = (uint32_t)(local % vw.spp);
      uint32_t k0 = vw.seedLo, k1 = vw.seedHi + vw.frame;
      int32_t hitPrim = -1;
      Draws dr;  // tape mode: one tape per path
      if (tapes) dr = Draws{tapes + pid * tape_len, 0, tape_len};
      U4 r0 = philox(U4{pixel, sample, 255u * 4u, vi}, k0, k1);
      const float jx = dr.take(u01(r0.x)), jy = dr.take(u01(r0.y));
      if ((vw.flags & VIEW_RESTIR) && !c.L.idx.empty() && c.L.total > 0.0f) {
        uint32_t px = pixel % vw.w, py = pixel / vw.w;
        float ux = ((float)px + 0.5f) / (float)vw.w, uy = ((float)py + 0.5f) / (float)vw.h;
        bool center = (vw.flags & 4u) != 0;
        float ss = ux + (center ? 0.0f : (jx - 0.5f) / (float)vw.w);
        float tt = uy + (center ? 0.0f : (jy - 0.5f) / (float)vw.h);
        V d = nrmz(v(vw.fp[0] + ss * vw.vu[0] + tt * vw.vv[0] - vw.cam[0], vw.fp[1] + ss * vw.vu[1] + tt * vw.vv[1] - vw.cam[1],
                    vw.fp[2] + ss * vw.vu[2] + tt * vw.vv[2] - vw.cam[2]));
        V o = v(vw.cam[0], vw.cam[1], vw.cam[2]);
        Hit h = closest(c, mkray(o, d, INFINITY));
        if (h.prim >= 0) {
          V p = v(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
          V n = geom_normal(prims, h.prim, p);
          if (!(dt(n, d) < 0.0f)) n = neg(n);
          Mat m = decode(materials, h.prim, view_lod(vw));
          if (lum(scl(m.diffuse, m.opacity)) > 0.0f) {
            V vd = nrmz(neg(d));
            V dd = vsub(p, o);
            s = SurfH{{p.x, p.y, p.z, std::sqrt(dt(dd, dd))}, {n.x, n.y, n.z, ibf(h.prim)}, {vd.x, vd.y, vd.z, 1.0f}};
            hitPrim = h.prim;
          }
        }
      }
      sCur[pid] = s;
      if (s.v[3] > 0.0f) {
        Mat m = decode(materials, hitPrim, view_lod(vw));
        for (uint32_t k = 0; k < C; ++k) {
          U4 u = philox(U4{pixel, sample, 0x10000u + k, vi}, k0, k1);
          uint32_t off = select_light(dr.take(u01(u.x)), c.L);
          int32_t lp = (int32_t)c.L.idx[off];
          if (lp == hitPrim) continue;
          V lpos, lnrm;
          float area = 0.0f;
          if (!light_point(prims, (uint32_t)lp, dr, u01(u.y), u01(u.z), lpos, lnrm, area) || !(area > 0.0f))
            continue;
          float lightPdf = light_pdf(c.L, off);
          Mat lm = decode(materials, lp, 1.0f);
          RefC cd;
          if (!ref_geometry(s, m, lpos, lnrm, 1.0f / area, lightPdf, scl(lm.emission, lm.power), lp, cd)) continue;
          refStats[tid][2]++;
          if (!ref_visible(c, s, cd)) continue;
          V cc = dvs(cd.radG, cd.pdf);
          float target = mx(lum(cd.radG), 0.0f);
          float w = cd.pdf > 0.0f ? target / cd.pdf : 0.0f;
          ref_update(r, contrib, cd, cc, w, 1.0f, dr, u01(u.w));
        }
        const float currentM = r.c[2];
        if (have_prev && temporal) {
          const View &pv = pvs[vi];
          // reuse candidate k (0..3: the pixel +x, -x, +y, -y; 4: the reprojected pixel)
          auto reuse = [&](uint32_t k, ResvH &q, int64_t &qid, bool &prevValid, RefC &cd) -> bool {
            qid = -1;
            prevValid = false;
            if (k < 4) {
              const int dx[4] = {1, -1, 0, 0}, dy[4] = {0, 0, 1, -1};
              int nx = (int)(pixel % vw.w) + dx[k], ny = (int)(pixel / vw.w) + dy[k];
              if (nx < 0 || ny < 0 || nx >= (int)pv.w || ny >= (int)pv.h) return false;
              qid = (int64_t)(poff[vi] + ((uint64_t)ny * pv.w + nx) * pv.spp + sample);
            } else if (g_vis_rule.load(std::memory_order_relaxed) & kRuleReprojection) {
              float m[16];
              oracle_vp::build(pv.cam, pv.vu, pv.vv, pv.fp, m);
              uint32_t ppx = 0, ppy = 0;
              if (!oracle_vp::reproject(m, s.p, pv.w, pv.h, ppx, ppy)) return false;
              qid = (int64_t)(poff[vi] + ((uint64_t)ppy * pv.w + ppx) * pv.spp + sample);
            } else {
              V cam = v(pv.cam[0], pv.cam[1], pv.cam[2]), U = v(pv.vu[0], pv.vu[1], pv.vu[2]);
              V Vv = v(pv.vv[0], pv.vv[1], pv.vv[2]), fp = v(pv.fp[0], pv.fp[1], pv.fp[2]);
              V pn = crs(U, Vv);
              V dd = vsub(v(s.p[0], s.p[1], s.p[2]), cam);
              float den = dt(dd, pn), num = dt(vsub(fp, cam), pn);
              if (den == 0.0f) return false;
              float lam = num / den;
              if (!(lam > 0.0f)) return false;
              V qq = add(cam, scl(dd, lam));
              V rel = vsub(qq, fp);
              float uu = dt(rel, U) / dt(U, U), ww = dt(rel, Vv) / dt(Vv, Vv);
              if (!(uu >= 0.0f && uu < 1.0f && ww >= 0.0f && ww < 1.0f)) return false;
              uint32_t ppx = std::min((uint32_t)(uu * (float)pv.w), pv.w - 1);
              uint32_t ppy = std::min((uint32_t)(ww * (float)pv.h), pv.h - 1);
              qid = (int64_t)(poff[vi] + ((uint64_t)ppy * pv.w + ppx) * pv.spp + sample);
            }
            if (!restir_gate(s, sPrev[qid])) return false;
            q = rPrev[qid];
            if (!(q.c[1] > 0.0f && q.c[2] > 0.0f && q.c[3] > 0.0f)) return false;
            prevValid = true;
            int32_t lp = fbi(q.a[3]);
            if (!(q.b[3] > 0.0f) || lp == hitPrim || lp < 0 || (uint32_t)lp >= prim_count) return false;
            Mat lm = decode(materials, lp, 1.0f);
            return ref_geometry(s, m, v(q.a[0], q.a[1], q.a[2]), v(q.b[0], q.b[1], q.b[2]), q.b[3], lpdfOf[lp],
                                scl(lm.emission, lm.power), lp, cd);
          };
          RefC rc[5];
          ResvH rq[5];
          int64_t rid[5];
          bool pvOk[5], cOk[5], visOk[5];
          for (uint32_t k = 0; k < 5; ++k) {
            cOk[k] = reuse(k, rq[k], rid[k], pvOk[k], rc[k]);
            visOk[k] = false;
            if (cOk[k]) {
              refStats[tid][2]++;
              visOk[k] = ref_visible(c, s, rc[k]);
            }
          }
          float totalSpatialM = 0.0f;
          for (uint32_t k = 0; k < 4; ++k)
            if (cOk[k] && visOk[k]) totalSpatialM = totalSpatialM + rq[k].c[2];
          for (uint32_t k = 0; k < 4; ++k) {
            if (!(cOk[k] && visOk[k])) continue;
            const RefC &cd = rc[k];
            const ResvH &q = rq[k];
            V cc = dvs(cd.radG, cd.pdf);
            float target = mx(lum(cd.radG), 0.0f);
            float prevTarget = q.c[3] * mx(q.c[0], RAY_EPS);
            float norm = q.c[2] > 0.0f ? q.c[1] / q.c[2] : 0.0f;
            float w = prevTarget > 0.0f ? norm * (target / prevTarget) : 0.0f;
            float sp = mx(cd.pdf, 0.0f);
            float den = sp * (currentM + totalSpatialM);
            if (pvOk[4]) den = den + rq[4].c[2] * sp * 1.0f;
            float mis = den > 0.0f ? (q.c[2] * sp) / den : 0.0f;
            w = w * mis;
            U4 rr = philox(U4{pixel, sample, 0x31000u + k, vi}, k0, k1);
            ref_update(r, contrib, cd, cc, w, q.c[2], dr, u01(rr.x));
          }
          if (pvOk[4] && cOk[4] && visOk[4]) {
            const RefC &cd = rc[4];
            const ResvH &q = rq[4];
            const SurfH &ps = sPrev[rid[4]];
            V cc = dvs(cd.radG, cd.pdf);
            float target = mx(lum(cd.radG), 0.0f);
            float prevTarget = q.c[3] * mx(cd.pdf, RAY_EPS);
            float norm = q.c[2] > 0.0f ? q.c[1] / q.c[2] : 0.0f;
            V toCur = vsub(cd.lpos, v(s.p[0], s.p[1], s.p[2])), toPrev = vsub(cd.lpos, v(ps.p[0], ps.p[1], ps.p[2]));
            float curD2 = mx(dt(toCur, toCur), RAY_EPS), prevD2 = mx(dt(toPrev, toPrev), RAY_EPS);
            V wiCur = nrmz(toCur), wiPrev = nrmz(toPrev);
            float cosCur = mx(dt(nrmz(v(s.n[0], s.n[1], s.n[2])), wiCur), 0.0f);
            float cosPrev = mx(dt(nrmz(nrmz(v(ps.n[0], ps.n[1], ps.n[2]))), wiPrev), 0.0f);
            float J = (prevD2 / curD2) * (cosCur / mx(cosPrev, RAY_EPS));
            if (!std::isfinite(J) || J < 0.0f) J = 0.0f;
            else J = mn(J, 32.0f);
            float w = prevTarget > 0.0f ? norm * (target / prevTarget) * J : 0.0f;
            float tp = mx(cd.pdf, 0.0f);
            float den = tp * (currentM + totalSpatialM);
            den = den + q.c[2] * tp * J;
            float mis = den > 0.0f ? (q.c[2] * tp * J) / den : 0.0f;
            w = w * mis;
            U4 rr = philox(U4{pixel, sample, 0x21000u, vi}, k0, k1);
            ref_update(r, contrib, cd, cc, w, q.c[2], dr, u01(rr.x));
          }
        }
        if (fbi(r.a[3]) >= 0 && r.c[3] > 0.0f && r.c[2] > 0.0f) {
          float norm = r.c[1] / (r.c[2] * r.c[3]);
          ro.valid = true;
          ro.direct = true;
          ro.contrib = scl(contrib, norm);
        }
      }
      ro.tapePos = dr.pos;
      rFin[pid] = r;
      roAll[pid] = ro;
    });
  }
  // initial
  if (!refMode) par([&](uint64_t pid, uint32_t) {
    uint32_t vi = view_of(pid);
    const View &vw = vs[vi];
    ResvH r = resv_empty();
    SurfH s{};
    uint64_t local = pid - poff[vi];
    uint32_t pixel = (uint32_t)(local / vw.spp), sample = (uint32_t)(local % vw.spp);
    uint32_t k0 = vw.seedLo, k1 = vw.seedHi + vw.frame;
    if ((vw.flags & VIEW_RESTIR) && !c.L.idx.empty() && c.L.total > 0.0f) {
      uint32_t px = pixel % vw.w, py = pixel / vw.w;
      U4 r0 = philox(U4{pixel, sample, 255u * 4u, vi}, k0, k1);
      float ux = ((float)px + 0.5f) / (float)vw.w, uy = ((float)py + 0.5f) / (float)vw.h;
      bool center = (vw.flags & 4u) != 0;
      float ss = ux + (center ? 0.0f : (u01(r0.x) - 0.5f) / (float)vw.w);
      float tt = uy + (center ? 0.0f : (u01(r0.y) - 0.5f) / (float)vw.h);
      V d = nrmz(v(vw.fp[0] + ss * vw.vu[0] + tt * vw.vv[0] - vw.cam[0], vw.fp[1] + ss * vw.vu[1] + tt * vw.vv[1] - vw.cam[1],
                  vw.fp[2] + ss * vw.vu[2] + tt * vw.vv[2] - vw.cam[2]));
      V o = v(vw.cam[0], vw.cam[1], vw.cam[2]);
      Hit h = closest(c, mkray(o, d, INFINITY));
      if (h.prim >= 0) {
        V p = v(o.x + h.t * d.x, o.y + h.t * d.y, o.z + h.t * d.z);
        V n = geom_normal(prims, h.prim, p);
        if (!(dt(n, d) < 0.0f)) n = neg(n);
        Mat m = decode(materials, h.prim, view_lod(vw));
        if (lum(scl(m.diffuse, m.opacity)) > 0.0f) {
          V vd = nrmz(neg(d));
          V dd = vsub(p, o);
          s = SurfH{{p.x, p.y, p.z, std::sqrt(dt(dd, dd))}, {n.x, n.y, n.z, ibf(h.prim)}, {vd.x, vd.y, vd.z, 1.0f}};
          for (uint32_t k = 0; k < C; ++k) {
            U4 u = philox(U4{pixel, sample, 0x10000u + k, vi}, k0, k1);
            uint32_t off = select_light(u01(u.x), c.L);
            int32_t lp = (int32_t)c.L.idx[off];
            V lpos{0, 0, 0}, lnrm{0, 0, 0};
            float area = 0.0f, w = 0.0f, ph = 0.0f;
            Draws slots;
            if (lp != h.prim && light_point(prims, (uint32_t)lp, slots, u01(u.y), u01(u.z), lpos, lnrm, area) &&
                area > 0.0f) {
              float prev = off > 0 ? c.L.cdf[off - 1] : 0.0f;
              float wgt = c.L.cdf[off] - prev;
              float lpdf = wgt > 0.0f ? wgt / c.L.total : 0.0f;
              float q = lpdf * (1.0f / area);
              V fa, wi;
              float dist;
              ph = restir_target(c, m, s, lpos, lnrm, lp, fa, wi, dist);
              w = q > 0.0f ? ph / q : 0.0f;
            }
            r.c[2] = r.c[2] + 1.0f;
            r.c[1] = r.c[1] + w;
            if (w > 0.0f && u01(u.w) * r.c[1] < w) {
              r.a[0] = lpos.x; r.a[1] = lpos.y; r.a[2] = lpos.z; r.a[3] = ibf(lp);
              r.b[0] = lnrm.x; r.b[1] = lnrm.y; r.b[2] = lnrm.z; r.b[3] = 0.0f;
              r.c[3] = ph;
            }
          }
        }
      }
    }
    rInit[pid] = r;
    sCur[pid] = s;
  });
  // temporal
  if (!refMode) par([&](uint64_t pid, uint32_t) {
    ResvH out = rInit[pid];
    const SurfH &s = sCur[pid];
    if (have_prev && temporal && s.v[3] > 0.0f) {
      uint32_t vi = view_of(pid);
      const View &vw = vs[vi], &pv = pvs[vi];
      V cam = v(pv.cam[0], pv.cam[1], pv.cam[2]), U = v(pv.vu[0], pv.vu[1], pv.vu[2]);
      V Vv = v(pv.vv[0], pv.vv[1], pv.vv[2]), fp = v(pv.fp[0], pv.fp[1], pv.fp[2]);
      V pn = crs(U, Vv);
      V dd = vsub(v(s.p[0], s.p[1], s.p[2]), cam);
      float den = dt(dd, pn), num = dt(vsub(fp, cam), pn);
      if (den != 0.0f) {
        float lam = num / den;
        if (lam > 0.0f) {
          V q = add(cam, scl(dd, lam));
          V rel = vsub(q, fp);
          float u = dt(rel, U) / dt(U, U), w = dt(rel, Vv) / dt(Vv, Vv);
          if (u >= 0.0f && u < 1.0f && w >= 0.0f && w < 1.0f) {
            uint32_t px = std::min((uint32_t)(u * (float)pv.w), pv.w - 1), py = std::min((uint32_t)(w * (float)pv.h), pv.h - 1);
            uint64_t local = pid - poff[vi];
            uint32_t pixel = (uint32_t)(local / vw.spp), sample = (uint32_t)(local % vw.spp);
            uint64_t ppid = poff[vi] + ((uint64_t)py * pv.w + px) * pv.spp + sample;
            if (restir_gate(s, sPrev[ppid])) {
              Mat m = decode(materials, fbi(s.n[3]), view_lod(vw));
              U4 rr = philox(U4{pixel, sample, 0x20000u, vi}, vw.seedLo, vw.seedHi + vw.frame);
              restir_merge(c, out, rPrev[ppid], s, m, capM, u01(rr.x));
            }
          }
        }
      }
    }
    rTemp[pid] = out;
  });
  // spatial
  if (!refMode) par([&](uint64_t pid, uint32_t) {
    ResvH out = rTemp[pid];
    const SurfH &s = sCur[pid];
    if (s.v[3] > 0.0f && spatialN > 0) {
      uint32_t vi = view_of(pid);
      const View &vw = vs[vi];
      uint64_t local = pid - poff[vi];
      uint32_t pixel = (uint32_t)(local / vw.spp), sample = (uint32_t)(local % vw.spp);
      int px = (int)(pixel % vw.w), py = (int)(pixel / vw.w);
      Mat m = decode(materials, fbi(s.n[3]), view_lod(vw));
      for (uint32_t k = 0; k < spatialN; ++k) {
        U4 rr = philox(U4{pixel, sample, 0x30000u + k, vi}, vw.seedLo, vw.seedHi + vw.frame);
        float rad = radius * std::sqrt(u01(rr.x));
        float sn, cs;
        sincos_turns(u01(rr.y), sn, cs);
        int nx = px + (int)std::floor(rad * cs + 0.5f), ny = py + (int)std::floor(rad * sn + 0.5f);
        if ((nx == px && ny == py) || nx < 0 || ny < 0 || nx >= (int)vw.w || ny >= (int)vw.h) continue;
        uint64_t npid = poff[vi] + ((uint64_t)ny * vw.w + nx) * vw.spp + sample;
        if (!restir_gate(s, sCur[npid])) continue;
        restir_merge(c, out, rTemp[npid], s, m, capM, u01(rr.z));
      }
    }
    rFin[pid] = out;
  });
  // final sample + the rest of each path
  std::vector<V> pathRad(P);
  std::vector<std::vector<uint64_t>> st(threads, std::vector<uint64_t>(4, 0));
  par([&](uint64_t pid, uint32_t tid) {
    uint32_t vi = view_of(pid);
    const View &vw = vs[vi];
    RestirOut ro;
    const ResvH &r = rFin[pid];
    const SurfH &s = sCur[pid];
    int32_t lp = fbi(r.a[3]);
    if (refMode) {
      ro = roAll[pid];
    } else if (s.v[3] > 0.0f && lp >= 0 && r.c[2] > 0.0f && r.c[1] > 0.0f && r.c[3] > 0.0f) {
      Mat m = decode(materials, fbi(s.n[3]), view_lod(vw));
      V fa, wi;
      float dist = 0.0f;
      float ph = restir_target(c, m, s, v(r.a[0], r.a[1], r.a[2]), v(r.b[0], r.b[1], r.b[2]), lp, fa, wi, dist);
      if (ph > 0.0f) {
        float W = r.c[1] / (r.c[2] * r.c[3]);
        ro.valid = true;
        ro.contrib = scl(fa, W);
        ro.tmax = dist - RAY_EPS;
        if (ro.tmax < RAY_EPS) ro.tmax = RAY_EPS;
        ro.origin = add(v(s.p[0], s.p[1], s.p[2]), scl(v(s.n[0], s.n[1], s.n[2]), 5.0f * RAY_EPS));
        ro.dir = wi;
      }
    }
    uint64_t local = pid - poff[vi];
    Draws dr;
    if (tapes) dr = Draws{tapes + pid * tape_len, 0, tape_len};
    pathRad[pid] = path(c, vw, vi, (uint32_t)(local / vw.spp), (uint32_t)(local % vw.spp), nullptr, st[tid].data(), &ro,
                        dr);
  });
  for (uint32_t vi = 0; vi < nviews; ++vi) {
    const View &vw = vs[vi];
    bool cl = (vw.flags & VIEW_CLAMP) != 0;
    for (uint64_t px = 0; px < (uint64_t)vw.w * vw.h; ++px) {
      float ax = 0.0f, ay = 0.0f, az = 0.0f;
      for (uint32_t sIdx = 0; sIdx < vw.spp; ++sIdx) {
        V r = pathRad[poff[vi] + px * vw.spp + sIdx];
        if (cl) r = v(c01(r.x), c01(r.y), c01(r.z));
        ax = ax + r.x;
        ay = ay + r.y;
        az = az + r.z;
      }
      float ns = (float)vw.spp;
      ax = ax / ns;
      ay = ay / ns;
      az = az / ns;
      if (cl) {
        ax = c01(ax);
        ay = c01(ay);
        az = c01(az);
      }
      float *o = out_rgb + 3 * (xoff[vi] + px);
      o[0] = ax;
      o[1] = ay;
      o[2] = az;
    }
  }
  if (stats) {
    for (auto &x : st)
      for (int k = 0; k < 4; ++k) stats[k] += x[k];
    for (auto &x : refStats)
      for (int k = 0; k < 4; ++k) stats[k] += x[k];
  }
  return 0;
}

}  // namespace

extern "C" int oracle_render_restir(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                                    const float *materials, const int32_t *prim_indices, const uint8_t *active,
                                    const int32_t *blas_root, const int32_t *prim_object, uint32_t object_count,
                                    uint32_t prim_count, const void *views, uint32_t nviews, const uint32_t *cfg_u,
                                    const float *cfg_f, const float *prev_resv, const float *prev_surf,
                                    const void *prev_views, int have_prev, float *out_resv, float *out_surf,
                                    float *out_rgb, uint64_t *stats, uint32_t threads) {
  return restir_impl(bvh, tlas, tlas_count, prims, materials, prim_indices, active, blas_root, prim_object,
                     object_count, prim_count, views, nviews, cfg_u, cfg_f, prev_resv, prev_surf, prev_views,
                     have_prev, out_resv, out_surf, out_rgb, stats, threads, nullptr, 0);
}

// oracle_render_restir in tape mode (reference mode only): `tapes` holds tape_len uniforms per
// path, drawn in the reference's order, for comparison with the reference's own rayColor run on
// the same numbers.
extern "C" int oracle_render_restir_tape(const float *bvh, const float *tlas, uint32_t tlas_count,
                                         const float *prims, const float *materials, const int32_t *prim_indices,
                                         const uint8_t *active, const int32_t *blas_root,
                                         const int32_t *prim_object, uint32_t object_count, uint32_t prim_count,
                                         const void *views, uint32_t nviews, const uint32_t *cfg_u,
                                         const float *cfg_f, const float *prev_resv, const float *prev_surf,
                                         const void *prev_views, int have_prev, float *out_resv, float *out_surf,
                                         float *out_rgb, uint64_t *stats, uint32_t threads, const float *tapes,
                                         uint32_t tape_len) {
  if (!tapes || tape_len == 0 || cfg_u[3] == 0) return 1;
  return restir_impl(bvh, tlas, tlas_count, prims, materials, prim_indices, active, blas_root, prim_object,
                     object_count, prim_count, views, nviews, cfg_u, cfg_f, prev_resv, prev_surf, prev_views,
                     have_prev, out_resv, out_surf, out_rgb, stats, threads, tapes, tape_len);
}

// ---------------------------------------------------------------------------------------------
// The functions above one at a time, for the pin against the reference's own functions
// (oracle/ref/ref_shade.cpp exports the reference's counterparts with the same arguments).
extern "C" {

// Light tables of the scene (build_lights: indices, CDF, total) and the per-primitive pdf.
// idx / cdf must hold prim_count entries; returns the light count.
uint32_t oracle_light_tables(const float *prims, const float *materials, const uint8_t *active,
                             const int32_t *blas_root, const int32_t *prim_object, uint32_t prim_count,
                             uint32_t *idx, float *cdf, float *total, float *pdf_of_prim) {
  LightsH L = build_lights(prims, materials, active, blas_root, prim_object, prim_count);
  std::copy(L.idx.begin(), L.idx.end(), idx);
  std::copy(L.cdf.begin(), L.cdf.end(), cdf);
  *total = L.total;
  std::vector<float> lk = light_pdf_lookup(L, prim_count);
  std::copy(lk.begin(), lk.end(), pdf_of_prim);
  return (uint32_t)L.idx.size();
}

// decode: per material 17 floats (decodeMaterial's numeric fields in ref_decode_material's order).
void oracle_decode_material(const float *mats, uint32_t n, float lod, float *out) {
  for (uint32_t i = 0; i < n; ++i) {
    Mat m = decode(mats, (int32_t)i, lod);
    const float vals[17] = {m.diffuse.x, m.diffuse.y, m.diffuse.z, m.opacity, m.specular.x, m.specular.y,
                            m.specular.z, m.shininess, m.emission.x, m.emission.y, m.emission.z, m.power,
                            m.transmission.x, m.transmission.y, m.transmission.z, m.ior, m.roughness};
    std::memcpy(out + 17ull * i, vals, sizeof(vals));
  }
}

void oracle_bsdf(const float *mats, const float *nvl, uint32_t n, float *out) {
  for (uint32_t i = 0; i < n; ++i) {
    Mat m = decode(mats, (int32_t)i, 1.0f);
    const float *q = nvl + 9ull * i;
    V f = bsdf(m, v(q[0], q[1], q[2]), v(q[3], q[4], q[5]), v(q[6], q[7], q[8]));
    out[3 * i] = f.x, out[3 * i + 1] = f.y, out[3 * i + 2] = f.z;
  }
}

void oracle_select_light(const float *xi, uint32_t n, const float *cdf, uint32_t count, float total, uint32_t *off,
                         float *pdf) {
  LightsH L;
  L.idx.assign(count, 0);
  L.cdf.assign(cdf, cdf + count);
  L.total = total;
  for (uint32_t i = 0; i < n; ++i) {
    off[i] = select_light(xi[i], L);
    pdf[i] = light_pdf(L, off[i]);
  }
}

void oracle_light_point(const float *prims, const float *uv, uint32_t n, float *out, uint8_t *ok) {
  for (uint32_t i = 0; i < n; ++i) {
    Draws dr{uv + 2ull * i, 0, 2};
    V p = v(0, 0, 0), nn = v(0, 0, 0);
    float area = 0.0f;
    ok[i] = light_point(prims, i, dr, 0.0f, 0.0f, p, nn, area) ? 1 : 0;
    const float vals[7] = {p.x, p.y, p.z, nn.x, nn.y, nn.z, area};
    std::memcpy(out + 7ull * i, vals, sizeof(vals));
  }
}

void oracle_scatter(const float *dn, const uint8_t *front, const float *mats, const float *tape4, uint32_t n,
                    float *out_dir, float *out_w, uint32_t *draws) {
  for (uint32_t i = 0; i < n; ++i) {
    Mat m = decode(mats, (int32_t)i, 1.0f);
    Draws dr{tape4 + 4ull * i, 0, 4};
    const float *q = dn + 6ull * i;
    V d = v(0, 0, 0);
    V w = scatter(v(q[0], q[1], q[2]), v(q[3], q[4], q[5]), front[i] != 0, m, dr, 0.0f, 0.0f, 0.0f, 0.0f, d);
    out_dir[3 * i] = d.x, out_dir[3 * i + 1] = d.y, out_dir[3 * i + 2] = d.z;
    out_w[3 * i] = w.x, out_w[3 * i + 1] = w.y, out_w[3 * i + 2] = w.z;
    draws[i] = dr.pos;
  }
}

// ref_update chains on ref_reservoir_chain's inputs; per chain 18 floats in its order, except
// that slot 7 holds the stored 1 / area and slot 3 the light id.
void oracle_reservoir_chain(const float *cand, const float *xi, uint32_t chains, uint32_t k, float *out) {
  for (uint32_t c = 0; c < chains; ++c) {
    ResvH r = resv_empty();
    V contrib = v(0, 0, 0);
    Draws dr{xi + (uint64_t)c * k, 0, k};
    for (uint32_t j = 0; j < k; ++j) {
      const float *q = cand + 16ull * ((uint64_t)c * k + j);
      RefC cd{v(q[0], q[1], q[2]), v(q[4], q[5], q[6]), v(0, 0, 0), scl(v(q[9], q[10], q[11]), q[12]),
              1.0f / q[7], 0.0f, q[8], (int32_t)q[3]};
      V cc = dvs(cd.radG, cd.pdf);
      float target = mx(lum(cd.radG), 0.0f);
      float w = (cd.pdf > 0.0f ? target / cd.pdf : 0.0f) * q[13];
      ref_update(r, contrib, cd, cc, w, q[14], dr, 0.0f);
    }
    const bool valid = fbi(r.a[3]) >= 0;
    const float vals[18] = {r.a[0], r.a[1], r.a[2], valid ? (float)fbi(r.a[3]) : 0.0f, r.b[0], r.b[1], r.b[2],
                            r.b[3], r.c[0], r.c[1], r.c[2], r.c[3], contrib.x, contrib.y, contrib.z,
                            valid ? 1.0f : 0.0f, (float)dr.pos, 0.0f};
    std::memcpy(out + 18ull * c, vals, sizeof(vals));
  }
}

}  // extern "C"

// Reference rules of the oracle's shading (bits kRuleVisibility, kRuleReprojection; 0 = the
// contract, the default); track != 0 also evaluates the other visibility rule on every light test
// and counts disagreements. Returns the counts since the last call (tests, decisions on which the
// two visibility rules differ) and resets them.
extern "C" void oracle_set_reference_rules(int rule, int track, uint64_t *counts) {
  g_vis_rule.store(rule);
  g_vis_track.store(track);
  if (counts) {
    counts[0] = g_vis_tests.exchange(0);
    counts[1] = g_vis_differ.exchange(0);
  }
}
