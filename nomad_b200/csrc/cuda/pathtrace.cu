// Wavefront path tracer: the reference's per-pixel rayColor loop (PathTracing.h:1069-1881,
// PathTraceKernel.metal:67-162) reorganised as stages over ray queues.
//
//   raygen  -> queue A (all paths of all views)
//   for each bounce:
//     trace closest (persistent warps over queue A)
//     shade: miss -> sky; hit -> counters, emission, one-sample NEE (shadow ray appended to
//            queue S with its unoccluded contribution), BSDF sample (ray appended to queue B)
//     trace any (persistent warps over queue S)
//     resolve: add the contribution of every unoccluded shadow ray
//     swap A and B
//   finalize: average the samples of each pixel (clamped to [0,1] per sample and per pixel when
//             NOMAD_VIEW_CLAMP, like pathTraceKernel)
//
// Queue appends are warp-aggregated (ballot + one atomic per warp). Every path owns fixed slots
// (throughput, radiance), so the order of a queue does not change any result, and the
// contributions of a path are added in the reference's order: emission, then direct light, per
// bounce. Random numbers come from Philox4x32-10 with key (seed_lo, seed_hi + frame) and counter
// (pixel, sample, 4*bounce + block, view): block 0 = (light choice, light u1, light u2, lobe
// choice), block 1 = (direction u1, direction u2, roulette, Fresnel choice); raygen uses bounce 255.
#include <algorithm>
#include <cstring>

#include "pt_lights.cuh"
#include "pt_math.cuh"
#include "rt_context.h"

using namespace nomad_dev;
using namespace nomad_pt;

namespace {

constexpr int kPtBlock = 256;
// Resident blocks per SM the ReSTIR candidate, spatial and reference-mode kernels are compiled
// for (a register cap): 4 was measured faster than 3, 5 and the uncapped build, same images.
#ifndef NOMAD_PT_MINB
#define NOMAD_PT_MINB 4
#endif
constexpr float kPi = 3.14159265358979323846f;

struct ViewDev {
  float cam[3], vu[3], vv[3], fp[3];
  float lod;
  uint32_t w, h, spp, maxDepth, k0, k1, flags, index;
  uint32_t tx, ty, tw;  // the rendered tile: origin and width in the view's pixels (0, 0, w: all)
  unsigned long long pathOffset, pixelOffset;
};

// The view pixel of the tile's pixel lp (row-major in the tile): the index that keys the path's
// random numbers and places its camera ray, so a tile's paths are the full view's paths.
__device__ __forceinline__ uint32_t tile_pixel(const ViewDev &v, uint32_t lp) {
  if (v.tw == v.w) return v.ty * v.w + lp;  // whole rows
  return (v.ty + lp / v.tw) * v.w + v.tx + lp % v.tw;
}

// Queue lengths 128 bytes apart: every warp of k_shade appends to the next-bounce and the shadow
// queue, and atomics to one cache line are serialised by one L2 slice.
constexpr int kQ = 32;
// Resident blocks per SM the shading kernel is compiled for: 4 (64 registers, about 110 bytes
// spilled) hides more of its dependent loads than 2 uncapped (105 registers) or 3 (80) did; the
// images are the same.
constexpr int kShadeMinBlocks = 4;
struct Counters {
  uint32_t qlen[4 * kQ];            // [kQ * k]: 0, 1 bounce queues; 2 shadow queue; 3 ReSTIR rays
  unsigned long long cursor[2];     // persistent-trace cursors (closest, any)
  unsigned long long stats[4];      // segments, escapes, shadow rays, hits
};

struct Lights {
  const uint32_t *idx;
  const float *cdf;
  const LightMeta *meta;
  const float4 *rec;  // per CDF slot, 5 float4 (pt_lights.cuh)
};

__device__ __forceinline__ const ViewDev &find_view(const ViewDev *views, uint32_t nviews,
                                                    unsigned long long pid) {
  uint32_t lo = 0, hi = nviews - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) / 2;
    if (views[mid].pathOffset <= pid) lo = mid;
    else hi = mid - 1;
  }
  return views[lo];
}

// Adds the sum of v over the warp's active lanes to *p with one atomic.
__device__ __forceinline__ void warp_sum64(unsigned long long *p, uint32_t v) {
  const unsigned act = __activemask();
  const uint32_t sum = __reduce_add_sync(act, v);
  if (sum && (threadIdx.x & 31) == __ffs(act) - 1) atomicAdd(p, (unsigned long long)sum);
}

// Warp-aggregated append: returns the slot of this lane (only meaningful when want).
__device__ __forceinline__ uint32_t warp_append(uint32_t *len, bool want) {
  unsigned act = __activemask();
  unsigned m = __ballot_sync(act, want);
  int lane = threadIdx.x & 31;
  int leader = __ffs(act) - 1;
  uint32_t base = 0;
  if (lane == leader && m) base = atomicAdd(len, (uint32_t)__popc(m));
  base = __shfl_sync(act, base, leader);
  return base + __popc(m & ((1u << lane) - 1u));
}

__global__ void __launch_bounds__(kPtBlock) k_raygen(const ViewDev *__restrict__ views, uint32_t nviews,
                                                      unsigned long long P, float4 *__restrict__ rays,
                                                      uint32_t *__restrict__ ids, float4 *__restrict__ thr,
                                                      float4 *__restrict__ rad, Counters *cnt) {
  unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long pid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; pid < P; pid += stride) {
    const ViewDev &v = find_view(views, nviews, pid);
    unsigned long long local = pid - v.pathOffset;
    uint32_t pixel = tile_pixel(v, (uint32_t)(local / v.spp)), sample = (uint32_t)(local % v.spp);
    uint32_t px = pixel % v.w, py = pixel / v.w;
    U4 r = philox(U4{pixel, sample, 255u * 4u, v.index}, v.k0, v.k1);
    float ux = ((float)px + 0.5f) / (float)v.w;
    float uy = ((float)py + 0.5f) / (float)v.h;
    bool center = (v.flags & NOMAD_VIEW_CENTER) != 0;
    float xo = center ? 0.0f : (u01(r.x) - 0.5f) / (float)v.w;
    float yo = center ? 0.0f : (u01(r.y) - 0.5f) / (float)v.h;
    float s = ux + xo, t = uy + yo;
    V3 d = v3(v.fp[0] + s * v.vu[0] + t * v.vv[0] - v.cam[0], v.fp[1] + s * v.vu[1] + t * v.vv[1] - v.cam[1],
              v.fp[2] + s * v.vu[2] + t * v.vv[2] - v.cam[2]);
    V3 dir = normalize(d);
    rays[2 * pid] = make_float4(v.cam[0], v.cam[1], v.cam[2], kRayEps);
    rays[2 * pid + 1] = make_float4(dir.x, dir.y, dir.z, INFINITY);
    ids[pid] = (uint32_t)pid;
    thr[pid] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    rad[pid] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt->qlen[kQ * (0)] = (uint32_t)P;
}

struct Material {
  V3 diffuse;
  float opacity;
  V3 specular;
  float shininess;
  V3 emission;
  float power;
  V3 transmission;
  float ior;
  float roughness;
};

// decodeMaterial (PathTracing.h:165-196), untextured.
__device__ __forceinline__ Material decode_material(const float4 *__restrict__ mats, int32_t prim, float lod) {
  const float4 *m = mats + 5ll * prim;
  float4 m0 = __ldg(m), m1 = __ldg(m + 1), m2 = __ldg(m + 2), m3 = __ldg(m + 3), m4 = __ldg(m + 4);
  Material o;
  o.diffuse = vmax0(ld3(m0) * lod);
  o.opacity = clamp01(m0.w);
  o.specular = vmax0(ld3(m1));
  o.shininess = fmax_ref(m1.w, 1.0f);
  o.emission = vmax0(ld3(m2));
  o.power = fmax_ref(m2.w, 0.0f);
  o.transmission = vmax0(ld3(m3));
  o.ior = fmax_ref(m3.w, 1e-3f);
  o.roughness = clamp01(m4.w);
  if (o.opacity < 1.0f && luminance(o.transmission) <= 0.0f) {
    float tr = 1.0f - o.opacity;
    o.transmission = v3(tr, tr, tr);
  }
  return o;
}

// The shading records and the material table, as the ReSTIR passes read them: a primitive's
// material is the table entry its record names (bits 0-29 of the record's w).
struct ShadeTables {
  const float4 *__restrict__ rec;
  const float4 *__restrict__ mat;
};

__device__ __forceinline__ Material prim_material(const ShadeTables &T, int32_t prim, float lod) {
  return decode_material(T.mat, (int32_t)(__float_as_uint(__ldg(T.rec + prim).w) & 0x3fffffffu), lod);
}

// Geometric normal at a hit, as firstHitBVH sets intersection.normal before the front-face flip
// (triangle :779-806, rectangle :853-863, sphere :766). For triangles and rectangles it does not
// depend on the hit point: surface_normal computes it from the primitive record alone.
__device__ __forceinline__ V3 surface_normal(int type, float4 p0, float4 p1, float4 p2, float4 p6) {
  V3 sn = ld3(p6);
  if (type == 1) {
    V3 e1 = ld3(p1) - ld3(p0), e2 = ld3(p2) - ld3(p0);
    V3 fb = cross(e1, e2);
    float fl = dot(fb, fb);
    fb = fl > 0.0f ? normalize(fb) : v3(0.0f, 1.0f, 0.0f);
    V3 n;
    float sl = dot(sn, sn);
    if (sl > kRayEps && finite3(sn)) n = normalize(sn);
    else n = fb;
    if (!finite3(n) || dot(n, n) <= kRayEps) n = fb;
    return n;
  }
  V3 fb = cross(ld3(p1), ld3(p2));
  float fl = dot(fb, fb);
  fb = (fl > kRayEps && finite3(fb)) ? normalize(fb) : v3(0.0f, 1.0f, 0.0f);
  float sl = dot(sn, sn);
  return (sl > kRayEps && finite3(sn)) ? normalize(sn) : fb;
}

// The compact shading record of a primitive: (normal, bits(material | type << 30)) for
// triangles and rectangles, (center, bits(material)) for spheres (type 0), whose normal is
// normalize(p - center) at the hit. 16 bytes gathered per hit instead of the 64 bytes of the
// primitive record and the 80 of its material.
constexpr uint32_t kShadeMatMask = 0x3fffffffu;

__device__ __forceinline__ V3 record_normal(float4 rec, V3 p) {
  return (__float_as_uint(rec.w) >> 30) == 0u ? normalize(p - ld3(rec)) : ld3(rec);
}

__global__ void k_shade_records(const float4 *__restrict__ prims, const uint32_t *__restrict__ matIdx, uint32_t n,
                                float4 *__restrict__ out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float4 *g = prims + 7ll * i;
  const float4 p0 = g[0];
  const int type = (int)p0.w;
  const uint32_t m = matIdx[i] & kShadeMatMask;
  if (type == 1 || type == 2) {
    const V3 nn = surface_normal(type, p0, g[1], g[2], g[6]);
    out[i] = make_float4(nn.x, nn.y, nn.z, __uint_as_float(m | ((uint32_t)type << 30)));
  } else {
    out[i] = make_float4(p0.x, p0.y, p0.z, __uint_as_float(m));
  }
}

// evaluateDirectLightingBsdf (PathTracing.h:249-293): Lambert + GGX D, Schlick-GGX G, Schlick F.
__device__ __forceinline__ V3 eval_bsdf(const Material &m, V3 normal, V3 viewDir, V3 lightDir) {
  V3 n = normalize(normal), v = normalize(viewDir), l = normalize(lightDir);
  if (!finite3(n) || !finite3(v) || !finite3(l)) return v3(0.0f, 0.0f, 0.0f);
  float nDotL = fmax_ref(dot(n, l), 0.0f), nDotV = fmax_ref(dot(n, v), 0.0f);
  if (nDotL <= 0.0f || nDotV <= 0.0f) return v3(0.0f, 0.0f, 0.0f);
  V3 diffuseColor = vmax0(m.diffuse) * m.opacity;
  V3 sc = m.specular * m.opacity;
  V3 specularColor = v3(clamp01(sc.x), clamp01(sc.y), clamp01(sc.z));
  float rough = clamp01(m.roughness);
  float alpha = fmax_ref(rough * rough, 0.001f);
  float alpha2 = alpha * alpha;
  V3 h = normalize(v + l);
  float nDotH = fmax_ref(dot(n, h), 0.0f), vDotH = fmax_ref(dot(v, h), 0.0f);
  float denom = nDotH * nDotH * (alpha2 - 1.0f) + 1.0f;
  float D = alpha2 / fmax_ref(kPi * denom * denom, kRayEps);
  float k = alpha + 1.0f;
  k = (k * k) / 8.0f;
  float Gv = nDotV / (nDotV * (1.0f - k) + k);
  float Gl = nDotL / (nDotL * (1.0f - k) + k);
  float G = Gv * Gl;
  float Fc = pow5(fmax_ref(1.0f - vDotH, 0.0f));
  V3 F = specularColor + (v3(1.0f, 1.0f, 1.0f) - specularColor) * Fc;
  V3 spec = F * (D * G) / fmax_ref(4.0f * nDotL * nDotV, kRayEps);
  V3 diff = diffuseColor / kPi;
  return diff + spec;
}

// buildOrthonormalBasis (Scatter.h:46-52).
__device__ __forceinline__ void onb(V3 n, V3 &t, V3 &b) {
  V3 up = fabsf(n.z) < 0.999f ? v3(0.0f, 0.0f, 1.0f) : v3(0.0f, 1.0f, 0.0f);
  t = normalize(cross(up, n));
  b = normalize(cross(n, t));
}

// scatter (Scatter.h:73-152). Returns the weight; writes the new direction.
__device__ __forceinline__ V3 scatter(V3 inDir, V3 normal, bool frontFace, const Material &m,
                                      float xiLobe, float u1, float u2, float xiFresnel, V3 &outDir) {
  float dw = fmax_ref(luminance(m.diffuse) * m.opacity, 0.0f);
  float sw = fmax_ref(luminance(m.specular) * m.opacity, 0.0f);
  float tw = fmax_ref(luminance(m.transmission) * (1.0f - m.opacity), 0.0f);
  if (tw > 0.0f) sw = 0.0f;
  float total = dw + sw + tw;
  if (total <= 0.0f) {
    outDir = normal;
    return v3(0.0f, 0.0f, 0.0f);
  }
  float xi = xiLobe * total;
  if (xi < dw) {
    // sampleCosineHemisphere (Scatter.h:54-71)
    float r = sqrtf(fmax_ref(0.0f, u1));
    float s, c;
    sincos_turns(u2, s, c);
    float x = r * c, y = r * s, z = sqrtf(fmax_ref(0.0f, 1.0f - u1));
    V3 t, b;
    onb(normal, t, b);
    outDir = normalize(t * x + b * y + normal * z);
    float prob = fmax_ref(dw / total, 1e-4f);
    return m.diffuse * m.opacity / prob;
  }
  xi = xi - dw;
  if (xi < sw) {
    V3 refl = reflect(inDir, normal);
    float exponent = fmax_ref(m.shininess, 1.0f);
    if (m.roughness > 0.0f) {
      float smooth = clamp01(1.0f - m.roughness);
      float re = fmax_ref(1.0f, smooth * smooth * 256.0f);
      exponent = fmax_ref(exponent, re);
    }
    float cosT = pow_pos(u1, 1.0f / (exponent + 1.0f));
    float sinT = sqrtf(fmax_ref(0.0f, 1.0f - cosT * cosT));
    float s, c;
    sincos_turns(u2, s, c);
    V3 t, b;
    onb(refl, t, b);
    outDir = normalize(t * (sinT * c) + b * (sinT * s) + refl * cosT);
    float prob = fmax_ref(sw / total, 1e-4f);
    return m.specular / prob;
  }
  float prob = fmax_ref(tw / total, 1e-4f);
  float eta = fmax_ref(m.ior, 1e-3f);
  float ratio = frontFace ? (1.0f / eta) : eta;
  // mirrorAngle (Scatter.h:31-44)
  float cosTheta = dot(-inDir, normal);
  float sinTheta = sqrtf(fmax_ref(0.0f, 1.0f - cosTheta * cosTheta));
  float r0 = (1.0f - ratio) / (1.0f + ratio);
  r0 = r0 * r0;
  float reflectance = r0 + (1.0f - r0) * pow5(1.0f - cosTheta);
  if ((ratio * sinTheta > 1.0f) || (reflectance > xiFresnel)) {
    outDir = reflect(inDir, normal);
    return m.specular / prob;
  }
  // refract (MSL definition): k = 1 - eta^2 (1 - dot(n,i)^2)
  float d = dot(normal, inDir);
  float k = 1.0f - ratio * ratio * (1.0f - d * d);
  if (k < 0.0f) {
    outDir = reflect(inDir, normal);
    return m.specular / prob;
  }
  V3 refr = inDir * ratio - normal * (ratio * d + sqrtf(k));
  if (!finite3(refr)) {
    outDir = reflect(inDir, normal);
    return m.specular / prob;
  }
  outDir = normalize(refr);
  return m.transmission / prob;
}

// sampleLightPoint (PathTracing.h:582-643).
// selectLightOffset (PathTracing.h:219-235).
__device__ __forceinline__ uint32_t select_light(float xi, const Lights &L, uint32_t count, float total) {
  float target = xi * total;
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (__ldg(L.cdf + mid) < target) lo = mid + 1;
    else hi = mid;
  }
  return lo < count - 1 ? lo : count - 1;
}

// The same search over a CDF copy (shared memory): the same predicate, so the same slot.
__device__ __forceinline__ uint32_t select_light_cdf(float xi, const float *cdf, uint32_t count, float total) {
  float target = xi * total;
  uint32_t lo = 0, hi = count;
  while (lo < hi) {
    uint32_t mid = (lo + hi) / 2;
    if (cdf[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  return lo < count - 1 ? lo : count - 1;
}

__global__ void __launch_bounds__(kPtBlock, kShadeMinBlocks) k_shade(
    uint32_t depth, const ViewDev *__restrict__ views, uint32_t nviews, const float4 *__restrict__ qRays,
    const uint32_t *__restrict__ qIds, const int32_t *__restrict__ hits, float4 *__restrict__ nRays,
    uint32_t *__restrict__ nIds, float4 *__restrict__ sRays, uint32_t *__restrict__ sIds,
    float4 *__restrict__ sContrib, float4 *__restrict__ thr, float4 *__restrict__ rad,
    const float4 *__restrict__ shadeRec, const float4 *__restrict__ matTable, Lights L, Counters *cnt, int cur,
    uint32_t *__restrict__ objHits, int restirDepth0, uint32_t *__restrict__ primHits) {
  const uint32_t n = cnt->qlen[kQ * (cur)];
  const uint32_t lightCount = L.meta->count;
  const float lightTotal = L.meta->total;
  uint32_t *nextLen = &cnt->qlen[kQ * (cur ^ 1)];
  uint32_t *shadowLen = &cnt->qlen[kQ * (2)];
  uint32_t stride = gridDim.x * blockDim.x;
  uint32_t iters = (n + stride - 1) / stride;
  // this thread's segments, escapes and hits, added to the frame's counters once at the end (one
  // atomic per warp and launch instead of three per warp and iteration on one cache line)
  uint32_t nSeg = 0, nEsc = 0, nHit = 0;
  for (uint32_t it = 0; it < iters; ++it) {
    uint32_t i = it * stride + blockIdx.x * blockDim.x + threadIdx.x;
    bool live = i < n;
    bool hit = false, wantShadow = false, wantNext = false;
    uint32_t pid = 0;
    float4 sA = make_float4(0, 0, 0, 0), sB = sA, sC = sA, nA = sA, nB = sA;
    int32_t inst = -1, hitPrim = -1;
    if (live) {
      pid = qIds[i];
      float4 ra = qRays[2 * i], rb = qRays[2 * i + 1];
      V3 o = ld3(ra), d = ld3(rb);
      const int32_t *h = hits + 5 * i;
      int32_t prim = h[1];
      hitPrim = prim;
      float t = __int_as_float(h[2]);
      float4 T = thr[pid];
      V3 tp = ld3(T);
      const ViewDev &v = find_view(views, nviews, pid);
      if (prim < 0) {
        // Sky (PathTracing.h:1211-1213): mix(1, (0.6, 0.7, 1.0), 0.5 (d.y + 1)).
        V3 ud = normalize(d);
        float s = 0.5f * (ud.y + 1.0f);
        V3 sky = v3(1.0f + (0.6f - 1.0f) * s, 1.0f + (0.7f - 1.0f) * s, 1.0f + (1.0f - 1.0f) * s);
        float4 R = rad[pid];
        rad[pid] = make_float4(R.x + tp.x * sky.x, R.y + tp.y * sky.y, R.z + tp.z * sky.z, R.w);
      } else {
        hit = true;
        inst = h[0];
        unsigned long long local = pid - v.pathOffset;
        uint32_t pixel = tile_pixel(v, (uint32_t)(local / v.spp)), sample = (uint32_t)(local % v.spp);
        U4 b0 = philox(U4{pixel, sample, depth * 4u + 0u, v.index}, v.k0, v.k1);
        U4 b1 = philox(U4{pixel, sample, depth * 4u + 1u, v.index}, v.k0, v.k1);
        V3 p = v3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
        const float4 rec = __ldg(shadeRec + prim);
        V3 nrm = record_normal(rec, p);
        bool front = dot(nrm, d) < 0.0f;
        if (!front) nrm = -nrm;
        Material m = decode_material(matTable, (int32_t)(__float_as_uint(rec.w) & kShadeMatMask), v.lod);
        float4 R = rad[pid];
        if (m.power * luminance(m.emission) > 0.0f) {
          R.x = R.x + tp.x * m.emission.x * m.power;
          R.y = R.y + tp.y * m.emission.y * m.power;
          R.z = R.z + tp.z * m.emission.z * m.power;
          rad[pid] = R;
        }
        V3 dc = m.diffuse * m.opacity;
        bool restirHere = restirDepth0 && depth == 0 && (v.flags & NOMAD_VIEW_RESTIR);
        if (!restirHere && luminance(dc) > 0.0f && lightCount > 0 && lightTotal > 0.0f) {
          uint32_t off = select_light(u01(b0.x), L, lightCount, lightTotal);
          // the light's sample-independent values come from its per-frame record
          const float4 *rec = L.rec + 5ull * off;
          const float4 r4 = __ldg(rec + 4);
          uint32_t lp = (uint32_t)__float_as_int(__ldg(rec + 3).w);
          if ((int32_t)lp != prim) {
            V3 lpos, lnrm;
            if (r4.w > 0.0f) {
              lpos = light_point(record_shape(rec), u01(b0.y), u01(b0.z), lnrm);
              V3 toL = lpos - p;
              float dist2 = dot(toL, toL);
              if (dist2 > kRayEps) {
                float dist = sqrtf(dist2);
                V3 wi = toL / dist;
                float cosT = fmax_ref(dot(nrm, wi), 0.0f);
                float cosL = fmax_ref(dot(lnrm, -wi), 0.0f);
                if (cosT > 0.0f && cosL > 0.0f) {
                  float lpdf = __ldg(rec).w;  // weight / total (lightTotal > 0 here)
                  if (lpdf > 0.0f) {
                    float pdfArea = __ldg(rec + 1).w;  // 1 / area
                    float pdfSolid = pdfArea * dist2 / cosL;
                    float totalPdf = lpdf * pdfSolid;
                    if (totalPdf > 0.0f) {
                      V3 lrad = ld3(r4);
                      V3 view = normalize(-d);
                      V3 bsdf = eval_bsdf(m, nrm, view, wi);
                      V3 c = tp * bsdf * lrad * (cosT / totalPdf);
                      // The reference accepts the light as visible when its closest hit is the
                      // light itself at t >= dist - 0.001 (PathTracing.h:1832-1834); a hit on the
                      // light a float rounding short of dist must not occlude it, so the any-hit
                      // window ends 1e-3 before the sampled point.
                      float tmax = dist - kNeeShadowEps;
                      if (tmax < kRayEps) tmax = kRayEps;
                      V3 so = p + nrm * 0.0005f;
                      sA = make_float4(so.x, so.y, so.z, kRayEps);
                      sB = make_float4(wi.x, wi.y, wi.z, tmax);
                      sC = make_float4(c.x, c.y, c.z, 0.0f);
                      wantShadow = true;
                    }
                  }
                }
              }
            }
          }
        }
        V3 nd;
        V3 wgt = scatter(d, nrm, front, m, u01(b0.w), u01(b1.x), u01(b1.y), u01(b1.w), nd);
        V3 bias = dot(nd, nrm) < 0.0f ? -nrm : nrm;
        V3 no = p + bias * kRayEps;
        V3 nt = tp * wgt;
        bool alive = true;
        if (depth >= 5) {
          float pm = fmax_ref(nt.x, fmax_ref(nt.y, nt.z));
          if (u01(b1.z) >= pm) alive = false;
          else nt = nt / pm;
        }
        thr[pid] = make_float4(nt.x, nt.y, nt.z, T.w);
        bool zero = nt.x == 0.0f && nt.y == 0.0f && nt.z == 0.0f;
        if (alive && !zero && depth + 1 < v.maxDepth) {
          nA = make_float4(no.x, no.y, no.z, kRayEps);
          nB = make_float4(nd.x, nd.y, nd.z, INFINITY);
          wantNext = true;
        }
      }
    }
    nSeg += live;
    nEsc += live && !hit;
    nHit += hit;
    // per-object (and per-primitive) closest hits, warp-aggregated by key
    if (objHits) {
      unsigned act = __activemask();
      int key = hit ? inst : -1;
      unsigned peers = __match_any_sync(act, key);
      if (hit && (threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(objHits + inst, (uint32_t)__popc(peers));
      if (primHits) {  // per-primitive closest hits (primitiveRayStats[2g], PathTracing.h:1216-1226)
        unsigned pp = __match_any_sync(act, hit ? hitPrim : -1);
        if (hit && (threadIdx.x & 31) == __ffs(pp) - 1) atomicAdd(primHits + hitPrim, (uint32_t)__popc(pp));
      }
    }
    uint32_t ss = warp_append(shadowLen, wantShadow);
    if (wantShadow) {
      sRays[2 * ss] = sA;
      sRays[2 * ss + 1] = sB;
      sIds[ss] = pid;
      sContrib[ss] = sC;
    }
    uint32_t ns = warp_append(nextLen, wantNext);
    if (wantNext) {
      nRays[2 * ns] = nA;
      nRays[2 * ns + 1] = nB;
      nIds[ns] = pid;
    }
  }
  warp_sum64(&cnt->stats[0], nSeg);
  warp_sum64(&cnt->stats[1], nEsc);
  warp_sum64(&cnt->stats[3], nHit);
}

__global__ void __launch_bounds__(kPtBlock) k_resolve(const uint32_t *__restrict__ sIds,
                                                       const float4 *__restrict__ sContrib,
                                                       const uint8_t *__restrict__ occ, float4 *__restrict__ rad,
                                                       Counters *cnt) {
  uint32_t n = cnt->qlen[kQ * (2)];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (occ[i]) continue;
    uint32_t pid = sIds[i];
    float4 c = sContrib[i], R = rad[pid];
    rad[pid] = make_float4(R.x + c.x, R.y + c.y, R.z + c.z, R.w);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt->stats[2] += n;
}

// Clears the next-bounce and shadow queue lengths and the trace cursors before a bounce.
__global__ void k_bounce_reset(Counters *cnt, int cur) {
  cnt->qlen[kQ * (cur ^ 1)] = 0;
  cnt->qlen[kQ * (2)] = 0;
  cnt->cursor[0] = 0;
  cnt->cursor[1] = 0;
}

__global__ void __launch_bounds__(kPtBlock) k_finalize(const ViewDev *__restrict__ views, uint32_t nviews,
                                                        unsigned long long totalPixels,
                                                        const float4 *__restrict__ rad, float *__restrict__ out) {
  for (unsigned long long q = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; q < totalPixels;
       q += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t lo = 0, hi = nviews - 1;
    while (lo < hi) {
      uint32_t mid = (lo + hi + 1) / 2;
      if (views[mid].pixelOffset <= q) lo = mid;
      else hi = mid - 1;
    }
    const ViewDev &v = views[lo];
    unsigned long long pixel = q - v.pixelOffset;
    bool clampOn = (v.flags & NOMAD_VIEW_CLAMP) != 0;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    for (uint32_t s = 0; s < v.spp; ++s) {
      float4 R = rad[v.pathOffset + pixel * v.spp + s];
      float x = R.x, y = R.y, z = R.z;
      if (clampOn) {
        x = clamp01(x);
        y = clamp01(y);
        z = clamp01(z);
      }
      ax = ax + x;
      ay = ay + y;
      az = az + z;
    }
    float ns = (float)v.spp;
    ax = ax / ns;
    ay = ay / ns;
    az = az / ns;
    if (clampOn) {
      ax = clamp01(ax);
      ay = clamp01(ay);
      az = clamp01(az);
    }
    out[3 * q + 0] = ax;
    out[3 * q + 1] = ay;
    out[3 * q + 2] = az;
  }
}

}  // namespace

// Builds the compact shading records at scene upload: the distinct 80-byte material records
// (compared bit for bit) go to a table, each primitive's record holds its table index, and the
// normal (or sphere center) is computed on the device by the same code the hit path used.
nomad_status nomad_build_shade_records(nomad_ctx *ctx, const float *materials, uint32_t primCount) {
  constexpr size_t kWords = 20;
  std::vector<uint32_t> idx(primCount);
  std::vector<float> table;
  {
    size_t cap = 1024;
    while (cap < 2ull * primCount) cap <<= 1;
    std::vector<int32_t> slots(cap, -1);
    for (uint32_t i = 0; i < primCount; ++i) {
      const float *m = materials + (size_t)i * kWords;
      uint32_t w[kWords];
      std::memcpy(w, m, sizeof(w));
      uint64_t h = 1469598103934665603ull;
      for (size_t k = 0; k < kWords; ++k) h = (h ^ w[k]) * 1099511628211ull;
      size_t at = (size_t)(h ^ (h >> 29)) & (cap - 1);
      while (true) {
        const int32_t e = slots[at];
        if (e < 0) {
          slots[at] = (int32_t)(table.size() / kWords);
          idx[i] = (uint32_t)slots[at];
          table.insert(table.end(), m, m + kWords);
          break;
        }
        if (std::memcmp(&table[(size_t)e * kWords], m, sizeof(w)) == 0) {
          idx[i] = (uint32_t)e;
          break;
        }
        at = (at + 1) & (cap - 1);
      }
    }
  }
  const uint32_t count = (uint32_t)(table.size() / kWords);
  if (count > kShadeMatMask) return nomad_fail(ctx, NOMAD_ERR_LIMIT, "more than 2^30 distinct materials");
  ctx->matCount = count;
  NOMAD_CUDA(ctx, ctx->matTable.reserve(std::max<size_t>(table.size() * 4, 80)));
  NOMAD_CUDA(ctx, ctx->shadeRec.reserve(std::max<size_t>((size_t)primCount * 16, 16)));
  if (primCount == 0) return NOMAD_OK;
  NOMAD_CUDA(ctx, cudaMemcpy(ctx->matTable.p, table.data(), table.size() * 4, cudaMemcpyHostToDevice));
  DeviceBuf d;
  NOMAD_CUDA(ctx, d.reserve((size_t)primCount * 4));
  NOMAD_CUDA(ctx, cudaMemcpy(d.p, idx.data(), (size_t)primCount * 4, cudaMemcpyHostToDevice));
  k_shade_records<<<(primCount + 255) / 256, 256, 0, ctx->stream>>>(ctx->prims.as<const float4>(),
                                                                    d.as<const uint32_t>(), primCount,
                                                                    ctx->shadeRec.as<float4>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_view_pinhole(const float pos[3], const float look[3], const float up[3],
                                           float vfov, uint32_t width, uint32_t height, nomad_view *out) {
  if (!pos || !look || !up || !out || width == 0 || height == 0 || !(vfov > 0.0f) || !(vfov < 180.0f))
    return NOMAD_ERR_INVALID_ARGUMENT;
  // populateViewportUniforms (Renderer.cpp:1237-1259).
  auto norm = [](float v[3]) {
    float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= l; v[1] /= l; v[2] /= l;
  };
  auto cross = [](const float a[3], const float b[3], float o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
  };
  float aspect = (float)width / (float)height;
  float fovRad = vfov * (3.14159265358979323846f / 180.0f);
  float halfH = std::tan(fovRad * 0.5f);
  float halfW = aspect * halfH;
  float fwd[3] = {look[0] - pos[0], look[1] - pos[1], look[2] - pos[2]};
  norm(fwd);
  float w[3] = {-fwd[0], -fwd[1], -fwd[2]};
  norm(w);
  float u[3], v[3];
  cross(up, w, u);
  norm(u);
  cross(w, u, v);
  std::memset(out, 0, sizeof(*out));
  for (int k = 0; k < 3; ++k) {
    out->camera_pos[k] = pos[k];
    out->viewport_u[k] = u[k] * (2.0f * halfW);
    out->viewport_v[k] = -v[k] * (2.0f * halfH);
  }
  for (int k = 0; k < 3; ++k)
    out->first_pixel[k] = pos[k] - w[k] - out->viewport_u[k] * 0.5f - out->viewport_v[k] * 0.5f;
  out->width = width;
  out->height = height;
  out->spp = 1;
  out->max_depth = 1;
  return NOMAD_OK;
}

namespace {
// ReSTIR state of one frame, fixed on the host before its kernels are launched or captured.
struct RestirPlan {
  bool on = false;
  int cur = 0;           // reservoir / surface buffers written this frame
  int temporal = 0;      // 1 when the previous frame's reservoirs are reused
  nomad_restir_config cfg{};
};
nomad_status restir_prepare(nomad_ctx *ctx, uint32_t nviews, const nomad_view *views, unsigned long long P,
                            RestirPlan &plan);
nomad_status restir_launch(nomad_ctx *ctx, uint32_t nviews, unsigned long long P, const Lights &L, Counters *C,
                           const RestirPlan &plan);
void restir_commit(nomad_ctx *ctx, uint32_t nviews, const nomad_view *views);

template <typename T>
void key_put(std::vector<unsigned char> &k, const T &v) {
  unsigned char b[sizeof(T)];
  std::memcpy(b, (const void *)&v, sizeof(T));
  k.insert(k.end(), b, b + sizeof(T));
}
}  // namespace

static nomad_status render_views(nomad_ctx *ctx, const nomad_view *views, const nomad_tile *tiles, uint32_t nviews,
                                 float *out, uint32_t flags);

extern "C" nomad_status nomad_render_frame(nomad_ctx *ctx, const nomad_view *views, uint32_t nviews,
                                           float *out, uint32_t flags) {
  return render_views(ctx, views, nullptr, nviews, out, flags);
}

extern "C" nomad_status nomad_render_tiles(nomad_ctx *ctx, const nomad_view *views, const nomad_tile *tiles,
                                           uint32_t nviews, float *out, uint32_t flags) {
  if (ctx && !tiles) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "no tiles");
  return render_views(ctx, views, tiles, nviews, out, flags);
}

// One frame over the views, each restricted to its tile when tiles is given (the whole view
// otherwise). Paths are numbered view by view and, in a view, by tile pixel and sample; the
// output holds each tile's pixels row-major, tile after tile.
static nomad_status render_views(nomad_ctx *ctx, const nomad_view *views, const nomad_tile *tiles, uint32_t nviews,
                                 float *out, uint32_t flags) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (!views || nviews == 0 || !out) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "no views or output");
  NOMAD_DEVICE_SCOPE(ctx);
  std::vector<ViewDev> vd(nviews);
  unsigned long long P = 0, pixels = 0;
  uint32_t maxDepth = 0;
  for (uint32_t i = 0; i < nviews; ++i) {
    const nomad_view &v = views[i];
    if (v.width == 0 || v.height == 0 || v.spp == 0 || v.max_depth == 0 || v.max_depth > 64)
      return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "view " + std::to_string(i) + " has a zero size, spp or depth");
    ViewDev &d = vd[i];
    for (int k = 0; k < 3; ++k) {
      d.cam[k] = v.camera_pos[k];
      d.vu[k] = v.viewport_u[k];
      d.vv[k] = v.viewport_v[k];
      d.fp[k] = v.first_pixel[k];
    }
    // Level-of-detail attenuation of the diffuse colour (PathTraceKernel.metal:78-81).
    float dx[3] = {v.viewport_u[0] / (float)v.width, v.viewport_u[1] / (float)v.width, v.viewport_u[2] / (float)v.width};
    float dy[3] = {v.viewport_v[0] / (float)v.height, v.viewport_v[1] / (float)v.height, v.viewport_v[2] / (float)v.height};
    float cx = dx[1] * dy[2] - dx[2] * dy[1], cy = dx[2] * dy[0] - dx[0] * dy[2], cz = dx[0] * dy[1] - dx[1] * dy[0];
    float fp = std::sqrt(cx * cx + cy * cy + cz * cz);
    d.lod = 1.0f / (1.0f + fp);
    d.w = v.width;
    d.h = v.height;
    d.spp = v.spp;
    d.maxDepth = v.max_depth;
    d.k0 = v.seed_lo;
    d.k1 = v.seed_hi + v.frame;
    d.flags = v.flags;
    d.index = i;
    uint32_t tw = v.width, th = v.height;
    d.tx = d.ty = 0;
    if (tiles) {
      const nomad_tile &t = tiles[i];
      if (t.width == 0 || t.height == 0 || t.origin_x >= v.width || t.origin_y >= v.height ||
          t.width > v.width - t.origin_x || t.height > v.height - t.origin_y)
        return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT,
                          "tile " + std::to_string(i) + " is empty or reaches outside its view");
      // ReSTIR's temporal and spatial reuse read the reservoirs of neighbouring pixels
      if ((v.flags & NOMAD_VIEW_RESTIR) && (t.width != v.width || t.height != v.height))
        return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT,
                          "view " + std::to_string(i) + " uses ReSTIR: its tile must be the whole view");
      d.tx = t.origin_x;
      d.ty = t.origin_y;
      tw = t.width;
      th = t.height;
    }
    d.tw = tw;
    d.pathOffset = P;
    d.pixelOffset = pixels;
    P += (unsigned long long)tw * th * v.spp;
    pixels += (unsigned long long)tw * th;
    maxDepth = std::max(maxDepth, v.max_depth);
  }
  if (P > 0xffffffffull) return nomad_fail(ctx, NOMAD_ERR_LIMIT, "more than 2^32 paths in one frame");
  FrameState &F = ctx->frame;
  nomad_status st = nomad_lights_update(ctx);
  if (st != NOMAD_OK) return st;
  if (F.capacity < P) {
    NOMAD_CUDA(ctx, F.thr.reserve(P * 16));
    NOMAD_CUDA(ctx, F.rad.reserve(P * 16));
    for (int k = 0; k < 2; ++k) {
      NOMAD_CUDA(ctx, F.qRays[k].reserve(P * 32));
      NOMAD_CUDA(ctx, F.qIds[k].reserve(P * 4));
    }
    NOMAD_CUDA(ctx, F.hits.reserve(P * 20));
    NOMAD_CUDA(ctx, F.sRays.reserve(P * 32));
    NOMAD_CUDA(ctx, F.sIds.reserve(P * 4));
    NOMAD_CUDA(ctx, F.sContrib.reserve(P * 16));
    NOMAD_CUDA(ctx, F.sOcc.reserve(P));
    F.capacity = P;
  }
  if (F.counters.bytes == 0) {
    NOMAD_CUDA(ctx, F.counters.reserve(sizeof(Counters)));
    NOMAD_CUDA(ctx, cudaMemset(F.counters.p, 0, sizeof(Counters)));
  }
  NOMAD_CUDA(ctx, F.views.reserve(nviews * sizeof(ViewDev)));
  cudaStream_t s = ctx->stream;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(F.views.p, vd.data(), nviews * sizeof(ViewDev), cudaMemcpyHostToDevice, s));
  // The view table is read by the kernels below; keep the host copy alive until they ran.
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));

  const ViewDev *V = F.views.as<const ViewDev>();
  Counters *C = F.counters.as<Counters>();
  Lights L{F.lightIdx.as<const uint32_t>(), F.lightCdf.as<const float>(), F.lightMeta.as<const LightMeta>(),
           F.lightRec.as<const float4>()};
  uint32_t *objHits = (flags & NOMAD_TRACE_COUNT_HITS) ? ctx->objHits.as<uint32_t>() : nullptr;
  uint32_t *primHits = (objHits && ctx->res.primHitsOn) ? ctx->res.primHits.as<uint32_t>() : nullptr;
  bool anyRestir = false;
  for (uint32_t i = 0; i < nviews; ++i) anyRestir |= (views[i].flags & NOMAD_VIEW_RESTIR) != 0;
  RestirPlan plan;
  if (anyRestir) {
    st = restir_prepare(ctx, nviews, views, P, plan);
    if (st != NOMAD_OK) return st;
  }
  float *dOut = out;
  bool hostOut = !(flags & NOMAD_TRACE_DEVICE_POINTERS);
  if (hostOut) {
    NOMAD_CUDA(ctx, ctx->stageAux.reserve(pixels * 12));
    dOut = ctx->stageAux.as<float>();
  }

  // The frame's device work: raygen, then per bounce closest hit, (ReSTIR at the first bounce),
  // shading, shadow any-hit and resolve, then the per-pixel average. Queue lengths stay on the
  // device, so the sequence needs no host synchronisation and can be captured as a graph.
  auto body = [&]() -> nomad_status {
    const int gridPT = ctx->smCount * 8;
    k_raygen<<<gridPT, kPtBlock, 0, s>>>(V, nviews, P, F.qRays[0].as<float4>(), F.qIds[0].as<uint32_t>(),
                                        F.thr.as<float4>(), F.rad.as<float4>(), C);
    NOMAD_CUDA(ctx, cudaGetLastError());
    int cur = 0;
    for (uint32_t depth = 0; depth < maxDepth; ++depth) {
      k_bounce_reset<<<1, 1, 0, s>>>(C, cur);
      nomad_status rs = nomad_trace_variant(ctx, ctx->trav, false, F.qRays[cur].as<const float4>(), P, &C->qlen[kQ * (cur)],
                                            &C->cursor[0], F.hits.as<int32_t>(), nullptr, nullptr, s);
      if (rs != NOMAD_OK) return rs;
      if (objHits && ctx->res.testsOn) {  // per-object "rays tested" for the hit posterior
        rs = nomad_count_object_tests(ctx, F.qRays[cur].as<const float4>(), F.hits.as<const int32_t>(), P,
                                      &C->qlen[kQ * (cur)]);
        if (rs != NOMAD_OK) return rs;
      }
      if (depth == 0 && plan.on) {
        rs = restir_launch(ctx, nviews, P, L, C, plan);
        if (rs != NOMAD_OK) return rs;
      }
      k_shade<<<gridPT, kPtBlock, 0, s>>>(depth, V, nviews, F.qRays[cur].as<const float4>(),
                                         F.qIds[cur].as<const uint32_t>(), F.hits.as<const int32_t>(),
                                         F.qRays[cur ^ 1].as<float4>(), F.qIds[cur ^ 1].as<uint32_t>(),
                                         F.sRays.as<float4>(), F.sIds.as<uint32_t>(), F.sContrib.as<float4>(),
                                         F.thr.as<float4>(), F.rad.as<float4>(), ctx->shadeRec.as<const float4>(),
                                         ctx->matTable.as<const float4>(), L, C, cur, objHits, plan.on ? 1 : 0,
                                         primHits);
      rs = nomad_trace_variant(ctx, ctx->trav, true, F.sRays.as<const float4>(), P, &C->qlen[kQ * (2)], &C->cursor[1],
                               nullptr, F.sOcc.as<uint8_t>(), nullptr, s);
      if (rs != NOMAD_OK) return rs;
      k_resolve<<<gridPT, kPtBlock, 0, s>>>(F.sIds.as<const uint32_t>(), F.sContrib.as<const float4>(),
                                           F.sOcc.as<const uint8_t>(), F.rad.as<float4>(), C);
      NOMAD_CUDA(ctx, cudaGetLastError());
      cur ^= 1;
    }
    k_finalize<<<gridPT, kPtBlock, 0, s>>>(V, nviews, pixels, F.rad.as<const float4>(), dOut);
    NOMAD_CUDA(ctx, cudaGetLastError());
    return NOMAD_OK;
  };

  if (flags & NOMAD_RENDER_DIRECT) {
    st = body();
    if (st != NOMAD_OK) return st;
  } else {
    // Everything the captured launches bake in: sizes, buffer addresses, kernel parameters.
    std::vector<unsigned char> key;
    key_put(key, nviews);
    key_put(key, P);
    key_put(key, pixels);
    key_put(key, maxDepth);
    key_put(key, objHits);
    key_put(key, primHits);
    key_put(key, ctx->res.testsOn);
    key_put(key, ctx->res.tests.p);
    key_put(key, ctx->res.tlas.p);
    key_put(key, dOut);
    key_put(key, ctx->trav);
    key_put(key, ctx->scene);
    for (const WideScene &w : ctx->ws) {
      key_put(key, w.wn);
      key_put(key, w.root);
    }
    key_put(key, ctx->smCount);
    key_put(key, ctx->res.emissiveCount);
    key_put(key, ctx->prims.p);
    key_put(key, ctx->materials.p);
    key_put(key, ctx->shadeRec.p);
    key_put(key, ctx->matTable.p);
    for (const DeviceBuf *b : {&F.thr, &F.rad, &F.qRays[0], &F.qRays[1], &F.qIds[0], &F.qIds[1], &F.hits, &F.sRays,
                               &F.sIds, &F.sContrib, &F.sOcc, &F.counters, &F.views, &F.lightIdx, &F.lightCdf,
                               &F.lightMeta, &F.rInit, &F.rTemp, &F.resv[0], &F.resv[1], &F.surf[0], &F.surf[1],
                               &F.prevViews, &F.lightPdf, &F.refRays, &F.refIds, &F.refOcc, &F.refMask,
                               &F.reuseMask, &F.refContrib})
      key_put(key, b->p);
    key_put(key, plan.on);
    key_put(key, plan.cur);
    key_put(key, plan.temporal);
    key_put(key, plan.cfg);
    FrameState::Graph *g = nullptr;
    for (FrameState::Graph &c : F.graphs)
      if (c.key == key) g = &c;
    if (!g) {
      constexpr size_t kMaxGraphs = 8;
      if (F.graphs.size() >= kMaxGraphs) {
        auto old = std::min_element(F.graphs.begin(), F.graphs.end(),
                                    [](const FrameState::Graph &a, const FrameState::Graph &b) { return a.lastUse < b.lastUse; });
        if (old->exec) cudaGraphExecDestroy(old->exec);
        if (old->graph) cudaGraphDestroy(old->graph);
        F.graphs.erase(old);
      }
      FrameState::Graph ng;
      ng.key = std::move(key);
      NOMAD_CUDA(ctx, cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      nomad_status cst = body();
      cudaError_t ce = cudaStreamEndCapture(s, &ng.graph);
      if (cst != NOMAD_OK) {
        if (ng.graph) cudaGraphDestroy(ng.graph);
        return cst;
      }
      if (ce != cudaSuccess) return nomad_cuda_fail(ctx, ce, "frame capture");
      ce = cudaGraphInstantiate(&ng.exec, ng.graph, 0);
      if (ce != cudaSuccess) {
        cudaGraphDestroy(ng.graph);
        return nomad_cuda_fail(ctx, ce, "frame graph instantiate");
      }
      ++F.graphCaptures;
      F.graphs.push_back(std::move(ng));
      g = &F.graphs.back();
    }
    g->lastUse = ++F.graphTick;
    NOMAD_CUDA(ctx, cudaGraphLaunch(g->exec, s));
    ++F.graphLaunches;
  }
  if (plan.on) restir_commit(ctx, nviews, views);
  if (hostOut) {
    NOMAD_CUDA(ctx, cudaMemcpyAsync(out, dOut, pixels * 12, cudaMemcpyDeviceToHost, s));
    NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  }
  return NOMAD_OK;
}

extern "C" nomad_status nomad_frame_graph_stats(nomad_ctx *ctx, uint64_t out[3]) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  out[0] = ctx->frame.graphCaptures;
  out[1] = ctx->frame.graphLaunches;
  out[2] = ctx->frame.graphs.size();
  return NOMAD_OK;
}

extern "C" nomad_status nomad_render_stats(nomad_ctx *ctx, uint64_t out[4]) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  std::memset(out, 0, 32);
  if (ctx->frame.counters.bytes == 0) return NOMAD_OK;
  Counters c;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(&c, ctx->frame.counters.p, sizeof(Counters), cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (int k = 0; k < 4; ++k) out[k] = c.stats[k];
  return NOMAD_OK;
}

extern "C" nomad_status nomad_reset_render_stats(nomad_ctx *ctx) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (ctx->frame.counters.bytes == 0) return NOMAD_OK;
  NOMAD_CUDA(ctx, cudaMemsetAsync(ctx->frame.counters.p, 0, sizeof(Counters), ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}


// ---------------------------------------------------------------------------------------------
// ReSTIR DI at the first bounce (views flagged NOMAD_VIEW_RESTIR).
//
// Per path (pixel, sample) the passes are:
//   initial  : RIS over `candidates` light samples (area measure: q(y) = lightPdf / area,
//              target p(y) = luminance(bsdf * Le * cos_theta * cos_light / dist^2), the
//              reference's luminance(radiance * geometryFactor), PathTracing.h:93-96, 383-394);
//   temporal : the previous frame's final reservoir at the reprojected pixel, gated by the
//              reference's surface tests (:1455-1473), its sample count capped at
//              m_cap * candidates, weight p_cur(y) * W_prev * M_prev;
//   spatial  : `spatial` neighbours within radius_px (Philox offsets) from this frame's temporal
//              reservoirs, same gates and weights;
//   shade    : W = wSum / (M * p(y)); the unoccluded contribution bsdf * Le * cos_theta *
//              cos_light / dist^2 * W is queued with one shadow ray (origin offset 5e-4 along the
//              normal, kVisibilityRayOffset :28), resolved with the other shadow rays.
// The reference weights candidates by target / (solid-angle pdf), which leaves a stray
// cos_light / dist^2 factor in its estimate; here the candidate pdf is in area measure, the
// measure the target is written in, so the estimate converges to the path-traced result and
// reuse across pixels needs no Jacobian.
namespace {

struct Resv {
  float4 a;  // light position, bits(light primitive) (-1: empty)
  float4 b;  // light normal, 0
  float4 c;  // 0, wSum, M, p(y) at the owner
};
struct Surf {
  float4 p;  // position, depth
  float4 n;  // shading normal, bits(primitive)
  float4 v;  // view direction, valid
};

struct RestirDev {
  uint32_t candidates, temporal, spatial;
  float radius, capM;
};

__device__ __forceinline__ Resv resv_empty() {
  Resv r;
  r.a = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(-1));
  r.b = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  r.c = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  return r;
}

// Unoccluded area-measure integrand at surface s for light point y; returns the target.
__device__ __forceinline__ float restir_target(const ShadeTables mats, const Material &m, const Surf &s,
                                               V3 lpos, V3 lnrm, int32_t lp, V3 &fa, V3 &wi, float &dist) {
  fa = v3(0.0f, 0.0f, 0.0f);
  if (lp < 0 || lp == __float_as_int(s.n.w)) return 0.0f;
  V3 p = ld3(s.p), n = ld3(s.n);
  V3 toL = lpos - p;
  float dist2 = dot(toL, toL);
  if (dist2 <= kRayEps) return 0.0f;
  dist = sqrtf(dist2);
  wi = toL / dist;
  float cosT = fmax_ref(dot(n, wi), 0.0f), cosL = fmax_ref(dot(lnrm, -wi), 0.0f);
  if (cosT <= 0.0f || cosL <= 0.0f) return 0.0f;
  Material lm = prim_material(mats, lp, 1.0f);
  V3 lrad = lm.emission * lm.power;
  V3 f = eval_bsdf(m, n, ld3(s.v), wi) * lrad * cosT;
  float g = cosL / fmax_ref(dist2, kRayEps);
  fa = f * g;
  return fmax_ref(luminance(fa), 0.0f);
}

// restir_target with the light's emitted radiance given (from its light record).
__device__ __forceinline__ float restir_target_rad(const Material &m, const Surf &s, V3 lpos, V3 lnrm, int32_t lp,
                                                   V3 lrad) {
  if (lp < 0 || lp == __float_as_int(s.n.w)) return 0.0f;
  V3 p = ld3(s.p), n = ld3(s.n);
  V3 toL = lpos - p;
  float dist2 = dot(toL, toL);
  if (dist2 <= kRayEps) return 0.0f;
  float dist = sqrtf(dist2);
  V3 wi = toL / dist;
  float cosT = fmax_ref(dot(n, wi), 0.0f), cosL = fmax_ref(dot(lnrm, -wi), 0.0f);
  if (cosT <= 0.0f || cosL <= 0.0f) return 0.0f;
  V3 f = eval_bsdf(m, n, ld3(s.v), wi) * lrad * cosT;
  float g = cosL / fmax_ref(dist2, kRayEps);
  V3 fa = f * g;
  return fmax_ref(luminance(fa), 0.0f);
}

__device__ __forceinline__ bool restir_gate(const Surf &s, const Surf &q) {
  if (q.v.w <= 0.0f) return false;
  float depth = s.p.w;
  V3 dp = ld3(q.p) - ld3(s.p);
  float posTh = fmax_ref(0.01f * depth, 0.02f), depTh = fmax_ref(0.02f * depth, 0.05f);
  if (!(length(dp) <= posTh)) return false;
  if (!(fabsf(q.p.w - depth) <= depTh)) return false;
  V3 qn = ld3(q.n);
  float qn2 = dot(qn, qn);
  if (!(qn2 > kRayEps)) return false;
  return dot(normalize(qn), normalize(ld3(s.n))) >= 0.9f;
}

// Adds a reused reservoir to `out` (the owner surface s, material m).
__device__ __forceinline__ void restir_merge(Resv &out, const Resv &src, const Surf &s, const Material &m,
                                             const ShadeTables mats, float capM, float u) {
  int32_t lp = __float_as_int(src.a.w);
  if (lp < 0 || !(src.c.z > 0.0f) || !(src.c.y > 0.0f) || !(src.c.w > 0.0f)) return;
  float Mp = fmin_ref(src.c.z, capM);
  float Wp = src.c.y / (src.c.z * src.c.w);
  V3 fa, wi;
  float dist;
  float ph = restir_target(mats, m, s, ld3(src.a), ld3(src.b), lp, fa, wi, dist);
  float w = ph * Wp * Mp;
  out.c.y = out.c.y + w;
  out.c.z = out.c.z + Mp;
  if (w > 0.0f && u * out.c.y < w) {
    out.a = src.a;
    out.b = src.b;
    out.c.w = ph;
  }
}

// The light CDF is staged in shared memory when it fits the block's allocation (cdfCap entries):
// every candidate binary-searches it, 32 per path.
__global__ void __launch_bounds__(kPtBlock, NOMAD_PT_MINB) k_restir_initial(
    const ViewDev *__restrict__ views, uint32_t nviews, unsigned long long P, RestirDev cfg,
    const float4 *__restrict__ rays, const int32_t *__restrict__ hits,
    const ShadeTables mats, Lights L, Resv *__restrict__ rOut, Surf *__restrict__ sOut, uint32_t cdfCap) {
  extern __shared__ float sCdf[];
  const uint32_t lightCount = L.meta->count;
  const float lightTotal = L.meta->total;
  const bool staged = lightCount <= cdfCap;
  if (staged)
    for (uint32_t i = threadIdx.x; i < lightCount; i += blockDim.x) sCdf[i] = L.cdf[i];
  __syncthreads();
  for (unsigned long long pid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; pid < P;
       pid += (unsigned long long)gridDim.x * blockDim.x) {
    const ViewDev &v = find_view(views, nviews, pid);
    Resv r = resv_empty();
    Surf s;
    s.p = s.n = s.v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const int32_t *h = hits + 5 * pid;
    int32_t prim = h[1];
    if ((v.flags & NOMAD_VIEW_RESTIR) && prim >= 0 && lightCount > 0 && lightTotal > 0.0f) {
      float t = __int_as_float(h[2]);
      V3 o = ld3(rays[2 * pid]), d = ld3(rays[2 * pid + 1]);
      V3 p = v3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
      V3 n = record_normal(__ldg(mats.rec + prim), p);
      if (!(dot(n, d) < 0.0f)) n = -n;
      Material m = prim_material(mats, prim, v.lod);
      if (luminance(m.diffuse * m.opacity) > 0.0f) {
        V3 vd = normalize(-d);
        s.p = make_float4(p.x, p.y, p.z, length(p - o));
        s.n = make_float4(n.x, n.y, n.z, __int_as_float(prim));
        s.v = make_float4(vd.x, vd.y, vd.z, 1.0f);
        unsigned long long local = pid - v.pathOffset;
        uint32_t pixel = (uint32_t)(local / v.spp), sample = (uint32_t)(local % v.spp);
        for (uint32_t c = 0; c < cfg.candidates; ++c) {
          U4 u = philox(U4{pixel, sample, 0x10000u + c, v.index}, v.k0, v.k1);
          uint32_t off = staged ? select_light_cdf(u01(u.x), sCdf, lightCount, lightTotal)
                                : select_light(u01(u.x), L, lightCount, lightTotal);
          // the light's sample-independent values come from its per-frame record
          const float4 *rec = L.rec + 5ull * off;
          const float4 r3 = __ldg(rec + 3), r4 = __ldg(rec + 4);
          int32_t lp = __float_as_int(r3.w);
          V3 lpos, lnrm;
          float w = 0.0f, ph = 0.0f;
          if (lp != prim && r4.w > 0.0f) {
            const LightShape sh = record_shape(rec);
            lpos = light_point(sh, u01(u.y), u01(u.z), lnrm);
            const float q = __ldg(rec + 2).w;
            ph = restir_target_rad(m, s, lpos, lnrm, lp, ld3(r4));
            w = q > 0.0f ? ph / q : 0.0f;
          }
          r.c.z = r.c.z + 1.0f;
          r.c.y = r.c.y + w;
          if (w > 0.0f && u01(u.w) * r.c.y < w) {
            r.a = make_float4(lpos.x, lpos.y, lpos.z, __int_as_float(lp));
            r.b = make_float4(lnrm.x, lnrm.y, lnrm.z, 0.0f);
            r.c.w = ph;
          }
        }
      }
    }
    rOut[pid] = r;
    sOut[pid] = s;
  }
}

__global__ void __launch_bounds__(kPtBlock) k_restir_temporal(
    const ViewDev *__restrict__ views, const ViewDev *__restrict__ prevViews, uint32_t nviews,
    unsigned long long P, RestirDev cfg, const ShadeTables mats, const Resv *__restrict__ rIn,
    const Surf *__restrict__ sCur, const Resv *__restrict__ rPrev, const Surf *__restrict__ sPrev,
    Resv *__restrict__ rOut, int usePrev) {
  for (unsigned long long pid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; pid < P;
       pid += (unsigned long long)gridDim.x * blockDim.x) {
    Resv out = rIn[pid];
    const Surf s = sCur[pid];
    if (usePrev && s.v.w > 0.0f) {
      const ViewDev &v = find_view(views, nviews, pid);
      const ViewDev &pv = prevViews[v.index];
      V3 cam = v3(pv.cam[0], pv.cam[1], pv.cam[2]), U = v3(pv.vu[0], pv.vu[1], pv.vu[2]);
      V3 Vv = v3(pv.vv[0], pv.vv[1], pv.vv[2]), fp = v3(pv.fp[0], pv.fp[1], pv.fp[2]);
      V3 pn = cross(U, Vv);
      V3 dd = ld3(s.p) - cam;
      float den = dot(dd, pn);
      float num = dot(fp - cam, pn);
      if (den != 0.0f) {
        float lam = num / den;
        if (lam > 0.0f) {
          V3 q = cam + dd * lam;
          V3 rel = q - fp;
          float u = dot(rel, U) / dot(U, U), w = dot(rel, Vv) / dot(Vv, Vv);
          if (u >= 0.0f && u < 1.0f && w >= 0.0f && w < 1.0f) {
            uint32_t px = min((uint32_t)(u * (float)pv.w), pv.w - 1), py = min((uint32_t)(w * (float)pv.h), pv.h - 1);
            unsigned long long local = pid - v.pathOffset;
            uint32_t pixel = (uint32_t)(local / v.spp), sample = (uint32_t)(local % v.spp);
            unsigned long long ppid = pv.pathOffset + ((unsigned long long)py * pv.w + px) * pv.spp + sample;
            if (restir_gate(s, sPrev[ppid])) {
              Material m = prim_material(mats, __float_as_int(s.n.w), v.lod);
              U4 rr = philox(U4{pixel, sample, 0x20000u, v.index}, v.k0, v.k1);
              restir_merge(out, rPrev[ppid], s, m, mats, cfg.capM * (float)cfg.candidates, u01(rr.x));
            }
          }
        }
      }
    }
    rOut[pid] = out;
  }
}

__global__ void __launch_bounds__(kPtBlock, NOMAD_PT_MINB) k_restir_spatial(
    const ViewDev *__restrict__ views, uint32_t nviews, unsigned long long P, RestirDev cfg,
    const ShadeTables mats, const Resv *__restrict__ rIn, const Surf *__restrict__ sCur,
    Resv *__restrict__ rOut) {
  for (unsigned long long pid = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; pid < P;
       pid += (unsigned long long)gridDim.x * blockDim.x) {
    Resv out = rIn[pid];
    const Surf s = sCur[pid];
    if (s.v.w > 0.0f && cfg.spatial > 0) {
      const ViewDev &v = find_view(views, nviews, pid);
      unsigned long long local = pid - v.pathOffset;
      uint32_t pixel = (uint32_t)(local / v.spp), sample = (uint32_t)(local % v.spp);
      int px = (int)(pixel % v.w), py = (int)(pixel / v.w);
      Material m = prim_material(mats, __float_as_int(s.n.w), v.lod);
      for (uint32_t k = 0; k < cfg.spatial; ++k) {
        U4 rr = philox(U4{pixel, sample, 0x30000u + k, v.index}, v.k0, v.k1);
        float rad = cfg.radius * sqrtf(u01(rr.x));
        float sn, cs;
        sincos_turns(u01(rr.y), sn, cs);
        int nx = px + (int)floorf(rad * cs + 0.5f), ny = py + (int)floorf(rad * sn + 0.5f);
        if ((nx == px && ny == py) || nx < 0 || ny < 0 || nx >= (int)v.w || ny >= (int)v.h) continue;
        unsigned long long npid = v.pathOffset + ((unsigned long long)ny * v.w + nx) * v.spp + sample;
        if (!restir_gate(s, sCur[npid])) continue;
        restir_merge(out, rIn[npid], s, m, mats, cfg.capM * (float)cfg.candidates, u01(rr.z));
      }
    }
    rOut[pid] = out;
  }
}

__global__ void __launch_bounds__(kPtBlock) k_restir_shade(
    const ViewDev *__restrict__ views, uint32_t nviews, unsigned long long P, const ShadeTables mats,
    const Resv *__restrict__ rIn, const Surf *__restrict__ sCur, float4 *__restrict__ sRays,
    uint32_t *__restrict__ sIds, float4 *__restrict__ sContrib, Counters *cnt) {
  unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  unsigned long long iters = (P + stride - 1) / stride;
  for (unsigned long long it = 0; it < iters; ++it) {
    unsigned long long pid = it * stride + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    float4 A = make_float4(0, 0, 0, 0), B = A, Cc = A;
    if (pid < P) {
      const Resv r = rIn[pid];
      const Surf s = sCur[pid];
      int32_t lp = __float_as_int(r.a.w);
      if (s.v.w > 0.0f && lp >= 0 && r.c.z > 0.0f && r.c.y > 0.0f && r.c.w > 0.0f) {
        const ViewDev &v = find_view(views, nviews, pid);
        Material m = prim_material(mats, __float_as_int(s.n.w), v.lod);
        V3 fa, wi;
        float dist = 0.0f;
        float ph = restir_target(mats, m, s, ld3(r.a), ld3(r.b), lp, fa, wi, dist);
        if (ph > 0.0f) {
          float W = r.c.y / (r.c.z * r.c.w);
          V3 c = fa * W;
          float tmax = dist - kRayEps;
          if (tmax < kRayEps) tmax = kRayEps;
          V3 o = ld3(s.p) + ld3(s.n) * (5.0f * kRayEps);
          A = make_float4(o.x, o.y, o.z, kRayEps);
          B = make_float4(wi.x, wi.y, wi.z, tmax);
          Cc = make_float4(c.x, c.y, c.z, 0.0f);
          want = true;
        }
      }
    }
    uint32_t slot = warp_append(&cnt->qlen[kQ * (2)], want);
    if (want) {
      sRays[2 * slot] = A;
      sRays[2 * slot + 1] = B;
      sIds[slot] = (uint32_t)pid;
      sContrib[slot] = Cc;
    }
  }
}

// ---- reference mode: the reference's own ReSTIR (PathTracing.h:308-480, :1363-1742) ----------
// Three passes around two visibility traces:
//   cand  : the surface record and every candidate's geometry (sampleDirectLightCandidate up to
//           its visibility test, :324-371); each surviving candidate queues its shadow ray;
//   reuse : RIS over the candidates whose ray was unoccluded (target / solid-angle pdf, :1393-
//           1398), then the reuse candidates of the previous frame (the reprojected pixel and
//           the 4 pixels +-1, gated as at :1455-1473 and :1531-1550) rebuilt from the stored
//           samples (buildRestirCandidateFromStored, :414-438), each queuing its shadow ray;
//   final : spatial then temporal resampling with the reference's MIS weights and Jacobian
//           (:1594-1706), the estimate weightSum / (M * selectedWeight) (:1708-1713), written to
//           the path through the shadow queue as an entry whose ray has an empty interval (so
//           it is added exactly where the configuration's estimate is).
// Reservoirs keep the reference's data0..data2 (:1716-1727): a = (light position, bits(light
// primitive)), b = (light normal, 1 / light area), c = (candidate pdf, weight sum, sample count,
// selected weight); the id is kept as an integer and the area as the reciprocal it is read as.

constexpr uint32_t kRefReuse = 5;  // 4 spatial neighbours (+x, -x, +y, -y) and the temporal sample

struct RefCand {
  V3 lpos, lnrm, wi, radG;  // radG = radiance * geometryFactor
  float invArea, dist, pdf;
  int32_t lp;
};

struct RefArgs {
  const float *lightPdf;  // per primitive (lightPdfLookup)
  uint32_t primCount;
  uint32_t words;         // candidate mask words per path
};

// Candidate geometry before its visibility test; false when the reference rejects it.
__device__ __forceinline__ bool ref_geometry(const Surf &s, const Material &m, V3 lpos, V3 lnrm, float invArea,
                                             float lightPdf, V3 lrad, int32_t lp, RefCand &c) {
  V3 p = ld3(s.p), n = ld3(s.n);
  V3 toL = lpos - p;
  float dist2 = dot(toL, toL);
  if (dist2 <= kRayEps) return false;
  float dist = sqrtf(dist2);
  V3 wi = toL / dist;
  float cosT = fmax_ref(dot(n, wi), 0.0f), cosL = fmax_ref(dot(lnrm, -wi), 0.0f);
  if (cosT <= 0.0f || cosL <= 0.0f) return false;
  if (lightPdf <= 0.0f) return false;
  float pdfSolid = invArea * dist2 / cosL;
  float pdf = lightPdf * pdfSolid;
  if (pdf <= 0.0f) return false;
  V3 rad = eval_bsdf(m, n, ld3(s.v), wi) * lrad * cosT;
  float g = cosL / fmax_ref(dist2, kRayEps);
  c.lpos = lpos;
  c.lnrm = lnrm;
  c.wi = wi;
  c.radG = rad * g;
  c.invArea = invArea;
  c.dist = dist;
  c.pdf = pdf;
  c.lp = lp;
  return true;
}

// New candidate c of a path (Philox stream 0x10000 + c, as in the configuration).
__device__ __forceinline__ bool ref_new_candidate(const Surf &s, const Material &m, const Lights &L, uint32_t lightCount,
                                                  float lightTotal, U4 u, RefCand &c) {
  const uint32_t off = select_light(u01(u.x), L, lightCount, lightTotal);
  const float4 *rec = L.rec + 5ull * off;
  const float4 r3 = __ldg(rec + 3), r4 = __ldg(rec + 4);
  const int32_t lp = __float_as_int(r3.w);
  if (lp == __float_as_int(s.n.w) || !(r4.w > 0.0f)) return false;
  V3 lnrm;
  const V3 lpos = light_point(record_shape(rec), u01(u.y), u01(u.z), lnrm);
  return ref_geometry(s, m, lpos, lnrm, __ldg(rec + 1).w, __ldg(rec).w, ld3(r4), lp, c);
}

// A candidate rebuilt from a stored reservoir sample.
__device__ __forceinline__ bool ref_stored_candidate(const Surf &s, const Material &m, const ShadeTables mats,
                                                     const RefArgs &ra, const Resv &src, RefCand &c) {
  const int32_t lp = __float_as_int(src.a.w);
  if (!(src.b.w > 0.0f) || lp == __float_as_int(s.n.w) || lp < 0 || (uint32_t)lp >= ra.primCount) return false;
  const Material lm = prim_material(mats, lp, 1.0f);
  return ref_geometry(s, m, ld3(src.a), ld3(src.b), src.b.w, ra.lightPdf[lp], lm.emission * lm.power, lp, c);
}

__device__ __forceinline__ bool ref_prev_valid(const Resv &q) {
  return q.c.y > 0.0f && q.c.z > 0.0f && q.c.w > 0.0f;
}

// restirUpdateReservoir (:98-115); `contrib` follows the selected sample.
__device__ __forceinline__ void ref_update(Resv &r, V3 &contrib, const RefCand &c, V3 cc, float w, float inc, float xi) {
  if (w <= 0.0f || inc <= 0.0f) return;
  r.c.y = r.c.y + w;
  r.c.z = r.c.z + inc;
  if (__float_as_int(r.a.w) < 0 || xi * r.c.y < w) {
    r.a = make_float4(c.lpos.x, c.lpos.y, c.lpos.z, __int_as_float(c.lp));
    r.b = make_float4(c.lnrm.x, c.lnrm.y, c.lnrm.z, c.invArea);
    r.c.x = c.pdf;
    r.c.w = w;
    contrib = cc;
  }
}

// The shadow ray of a candidate (isLightVisible, :511-521): origin offset 5e-4 along the normal.
__device__ __forceinline__ void ref_ray(const Surf &s, const RefCand &c, float4 &A, float4 &B) {
  V3 o = ld3(s.p) + ld3(s.n) * (5.0f * kRayEps);
  float tmax = c.dist - kRayEps;
  if (tmax < kRayEps) tmax = kRayEps;
  A = make_float4(o.x, o.y, o.z, kRayEps);
  B = make_float4(c.wi.x, c.wi.y, c.wi.z, tmax);
}

// The previous frame's path at the pixel this path's surface reprojects to, or -1.
__device__ __forceinline__ long long ref_reproject(const ViewDev &v, const ViewDev &pv, const Surf &s, uint32_t sample) {
  V3 cam = v3(pv.cam[0], pv.cam[1], pv.cam[2]), U = v3(pv.vu[0], pv.vu[1], pv.vu[2]);
  V3 Vv = v3(pv.vv[0], pv.vv[1], pv.vv[2]), fp = v3(pv.fp[0], pv.fp[1], pv.fp[2]);
  V3 pn = cross(U, Vv);
  V3 dd = ld3(s.p) - cam;
  float den = dot(dd, pn);
  float num = dot(fp - cam, pn);
  if (den == 0.0f) return -1;
  float lam = num / den;
  if (!(lam > 0.0f)) return -1;
  V3 q = cam + dd * lam;
  V3 rel = q - fp;
  float u = dot(rel, U) / dot(U, U), w = dot(rel, Vv) / dot(Vv, Vv);
  if (!(u >= 0.0f && u < 1.0f && w >= 0.0f && w < 1.0f)) return -1;
  uint32_t px = min((uint32_t)(u * (float)pv.w), pv.w - 1), py = min((uint32_t)(w * (float)pv.h), pv.h - 1);
  return (long long)(pv.pathOffset + ((unsigned long long)py * pv.w + px) * pv.spp + sample);
}

// The previous frame's path at neighbour k (0..3: +x, -x, +y, -y) of this path's pixel, or -1.
__device__ __forceinline__ long long ref_neighbour(const ViewDev &v, const ViewDev &pv, uint32_t pixel, uint32_t sample,
                                                   uint32_t k) {
  const int dx[4] = {1, -1, 0, 0}, dy[4] = {0, 0, 1, -1};
  int nx = (int)(pixel % v.w) + dx[k], ny = (int)(pixel / v.w) + dy[k];
  if (nx < 0 || ny < 0 || nx >= (int)pv.w || ny >= (int)pv.h) return -1;
  return (long long)(pv.pathOffset + ((unsigned long long)ny * pv.w + nx) * pv.spp + sample);
}

// Reuse candidate k of a path: the prior reservoir it comes from and the rebuilt candidate.
__device__ __forceinline__ bool ref_reuse_candidate(uint32_t k, const ViewDev &v, const ViewDev &pv, const Surf &s,
                                                    const Material &m, const ShadeTables mats,
                                                    const RefArgs &ra, const Resv *__restrict__ rPrev,
                                                    const Surf *__restrict__ sPrev, uint32_t pixel, uint32_t sample,
                                                    Resv &q, long long &qid, bool &prevValid, RefCand &c) {
  qid = k < 4 ? ref_neighbour(v, pv, pixel, sample, k) : ref_reproject(v, pv, s, sample);
  prevValid = false;
  if (qid < 0 || !restir_gate(s, sPrev[qid])) return false;
  q = rPrev[qid];
  if (!ref_prev_valid(q)) return false;
  prevValid = true;
  return ref_stored_candidate(s, m, mats, ra, q, c);
}

__global__ void __launch_bounds__(kPtBlock, NOMAD_PT_MINB) k_restir_ref_cand(
    const ViewDev *__restrict__ views, uint32_t nviews, unsigned long long P, RestirDev cfg,
    const float4 *__restrict__ rays, const int32_t *__restrict__ hits,
    const ShadeTables mats, Lights L, Surf *__restrict__ sOut, uint32_t *__restrict__ mask, RefArgs ra,
    float4 *__restrict__ qRays, uint32_t *__restrict__ qIds, Counters *cnt) {
  const uint32_t lightCount = L.meta->count;
  const float lightTotal = L.meta->total;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long iters = (P + stride - 1) / stride;
  for (unsigned long long it = 0; it < iters; ++it) {
    const unsigned long long pid = it * stride + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    Surf s;
    s.p = s.n = s.v = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    Material m{};
    uint32_t pixel = 0, sample = 0;
    const ViewDev *vp = nullptr;
    if (pid < P) {
      const ViewDev &v = find_view(views, nviews, pid);
      vp = &v;
      const int32_t *h = hits + 5 * pid;
      const int32_t prim = h[1];
      if ((v.flags & NOMAD_VIEW_RESTIR) && prim >= 0 && lightCount > 0 && lightTotal > 0.0f) {
        float t = __int_as_float(h[2]);
        V3 o = ld3(rays[2 * pid]), d = ld3(rays[2 * pid + 1]);
        V3 p = v3(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
        V3 n = record_normal(__ldg(mats.rec + prim), p);
        if (!(dot(n, d) < 0.0f)) n = -n;
        m = prim_material(mats, prim, v.lod);
        if (luminance(m.diffuse * m.opacity) > 0.0f) {
          V3 vd = normalize(-d);
          s.p = make_float4(p.x, p.y, p.z, length(p - o));
          s.n = make_float4(n.x, n.y, n.z, __int_as_float(prim));
          s.v = make_float4(vd.x, vd.y, vd.z, 1.0f);
        }
      }
      unsigned long long local = pid - v.pathOffset;
      pixel = (uint32_t)(local / v.spp);
      sample = (uint32_t)(local % v.spp);
      sOut[pid] = s;
      for (uint32_t w = 0; w < ra.words; ++w) mask[pid * ra.words + w] = 0u;
    }
    for (uint32_t c = 0; c < cfg.candidates; ++c) {
      RefCand cd;
      bool want = false;
      if (s.v.w > 0.0f) {
        const U4 u = philox(U4{pixel, sample, 0x10000u + c, vp->index}, vp->k0, vp->k1);
        want = ref_new_candidate(s, m, L, lightCount, lightTotal, u, cd);
      }
      const uint32_t slot = warp_append(&cnt->qlen[kQ * (3)], want);
      if (want) {
        float4 A, B;
        ref_ray(s, cd, A, B);
        qRays[2ull * slot] = A;
        qRays[2ull * slot + 1] = B;
        qIds[slot] = (uint32_t)(pid * cfg.candidates + c);
      }
    }
  }
}

// Unoccluded entries of the visibility queue set their bit in the path's mask.
__global__ void __launch_bounds__(kPtBlock) k_restir_ref_vis(const uint32_t *__restrict__ ids,
                                                             const uint8_t *__restrict__ occ, uint32_t per,
                                                             uint32_t words, uint32_t *__restrict__ mask,
                                                             Counters *cnt) {
  const uint32_t n = cnt->qlen[kQ * (3)];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (occ[i]) continue;
    const uint32_t id = ids[i], pid = id / per, c = id - pid * per;
    atomicOr(&mask[(unsigned long long)pid * words + c / 32], 1u << (c % 32));
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt->stats[2] += n;
}

__global__ void k_restir_ref_reset(Counters *cnt) {
  cnt->qlen[kQ * (3)] = 0;
  cnt->cursor[1] = 0;
}

__global__ void __launch_bounds__(kPtBlock, NOMAD_PT_MINB) k_restir_ref_reuse(
    const ViewDev *__restrict__ views, const ViewDev *__restrict__ prevViews, uint32_t nviews, unsigned long long P,
    RestirDev cfg, const ShadeTables mats, Lights L, const Surf *__restrict__ sCur,
    const uint32_t *__restrict__ candMask, RefArgs ra, const Resv *__restrict__ rPrev, const Surf *__restrict__ sPrev,
    int usePrev, Resv *__restrict__ rMid, float4 *__restrict__ midContrib, uint32_t *__restrict__ reuseMask,
    float4 *__restrict__ qRays, uint32_t *__restrict__ qIds, Counters *cnt) {
  const uint32_t lightCount = L.meta->count;
  const float lightTotal = L.meta->total;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long iters = (P + stride - 1) / stride;
  for (unsigned long long it = 0; it < iters; ++it) {
    const unsigned long long pid = it * stride + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    Surf s;
    s.v.w = 0.0f;
    Material m{};
    uint32_t pixel = 0, sample = 0;
    const ViewDev *vp = nullptr;
    if (pid < P) {
      s = sCur[pid];
      const ViewDev &v = find_view(views, nviews, pid);
      vp = &v;
      unsigned long long local = pid - v.pathOffset;
      pixel = (uint32_t)(local / v.spp);
      sample = (uint32_t)(local % v.spp);
      Resv r = resv_empty();
      V3 contrib = v3(0.0f, 0.0f, 0.0f);
      if (s.v.w > 0.0f) {
        m = prim_material(mats, __float_as_int(s.n.w), v.lod);
        for (uint32_t c = 0; c < cfg.candidates; ++c) {
          if (!((candMask[pid * ra.words + c / 32] >> (c % 32)) & 1u)) continue;
          const U4 u = philox(U4{pixel, sample, 0x10000u + c, v.index}, v.k0, v.k1);
          RefCand cd;
          if (!ref_new_candidate(s, m, L, lightCount, lightTotal, u, cd)) continue;
          const V3 cc = cd.radG / cd.pdf;
          const float target = fmax_ref(luminance(cd.radG), 0.0f);
          const float w = cd.pdf > 0.0f ? target / cd.pdf : 0.0f;
          ref_update(r, contrib, cd, cc, w, 1.0f, u01(u.w));
        }
      }
      rMid[pid] = r;
      midContrib[pid] = make_float4(contrib.x, contrib.y, contrib.z, 0.0f);
      reuseMask[pid] = 0u;
    }
    for (uint32_t k = 0; k < kRefReuse; ++k) {
      RefCand cd;
      bool want = false;
      if (usePrev && s.v.w > 0.0f) {
        Resv q;
        long long qid;
        bool pv;
        want = ref_reuse_candidate(k, *vp, prevViews[vp->index], s, m, mats, ra, rPrev, sPrev, pixel, sample, q, qid,
                                   pv, cd);
      }
      const uint32_t slot = warp_append(&cnt->qlen[kQ * (3)], want);
      if (want) {
        float4 A, B;
        ref_ray(s, cd, A, B);
        qRays[2ull * slot] = A;
        qRays[2ull * slot + 1] = B;
        qIds[slot] = (uint32_t)(pid * kRefReuse + k);
      }
    }
  }
}

__global__ void __launch_bounds__(kPtBlock, NOMAD_PT_MINB) k_restir_ref_final(
    const ViewDev *__restrict__ views, const ViewDev *__restrict__ prevViews, uint32_t nviews, unsigned long long P,
    const ShadeTables mats, const Surf *__restrict__ sCur, RefArgs ra, const Resv *__restrict__ rPrev,
    const Surf *__restrict__ sPrev, int usePrev, const Resv *__restrict__ rMid, const float4 *__restrict__ midContrib,
    const uint32_t *__restrict__ reuseMask, Resv *__restrict__ rOut, float4 *__restrict__ sRays,
    uint32_t *__restrict__ sIds, float4 *__restrict__ sContrib, Counters *cnt) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  const unsigned long long iters = (P + stride - 1) / stride;
  for (unsigned long long it = 0; it < iters; ++it) {
    const unsigned long long pid = it * stride + (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    bool want = false;
    float4 A = make_float4(0, 0, 0, 0), B = A, Cc = A;
    if (pid < P) {
      const Surf s = sCur[pid];
      Resv r = rMid[pid];
      if (s.v.w > 0.0f) {
        const ViewDev &v = find_view(views, nviews, pid);
        const unsigned long long local = pid - v.pathOffset;
        const uint32_t pixel = (uint32_t)(local / v.spp), sample = (uint32_t)(local % v.spp);
        const Material m = prim_material(mats, __float_as_int(s.n.w), v.lod);
        const float4 mc = midContrib[pid];
        V3 contrib = v3(mc.x, mc.y, mc.z);
        const float currentM = r.c.z;
        const uint32_t vis = reuseMask[pid];
        if (usePrev) {
          const ViewDev &pv = prevViews[v.index];
          // temporal validity (the gate and a usable prior reservoir), needed by the spatial MIS
          Resv tq;
          long long tqid;
          bool tPrevValid = false;
          RefCand tc;
          const bool tCand = ref_reuse_candidate(4, v, pv, s, m, mats, ra, rPrev, sPrev, pixel, sample, tq, tqid,
                                                 tPrevValid, tc);
          // spatial candidates that survived their visibility test (:1531-1591)
          RefCand sc[4];
          Resv sq[4];
          bool sOk[4];
          float totalSpatialM = 0.0f;
          for (uint32_t k = 0; k < 4; ++k) {
            long long qid;
            bool pvv;
            sOk[k] = ref_reuse_candidate(k, v, pv, s, m, mats, ra, rPrev, sPrev, pixel, sample, sq[k], qid, pvv,
                                         sc[k]) &&
                     ((vis >> k) & 1u);
            if (sOk[k]) totalSpatialM = totalSpatialM + sq[k].c.z;
          }
          for (uint32_t k = 0; k < 4; ++k) {
            if (!sOk[k]) continue;
            const RefCand &c = sc[k];
            const Resv &q = sq[k];
            const V3 cc = c.radG / c.pdf;
            const float target = fmax_ref(luminance(c.radG), 0.0f);
            const float prevTarget = q.c.w * fmax_ref(q.c.x, kRayEps);
            const float norm = q.c.z > 0.0f ? q.c.y / q.c.z : 0.0f;
            float w = prevTarget > 0.0f ? norm * (target / prevTarget) : 0.0f;
            const float sp = fmax_ref(c.pdf, 0.0f);
            float den = sp * (currentM + totalSpatialM);
            if (tPrevValid) den = den + tq.c.z * sp * 1.0f;
            const float mis = den > 0.0f ? (q.c.z * sp) / den : 0.0f;
            w = w * mis;
            const U4 rr = philox(U4{pixel, sample, 0x31000u + k, v.index}, v.k0, v.k1);
            ref_update(r, contrib, c, cc, w, q.c.z, u01(rr.x));
          }
          // temporal (:1633-1706)
          if (tPrevValid && tCand && ((vis >> 4) & 1u)) {
            const RefCand &c = tc;
            const V3 cc = c.radG / c.pdf;
            const float target = fmax_ref(luminance(c.radG), 0.0f);
            const float prevTarget = tq.c.w * fmax_ref(c.pdf, kRayEps);
            const float norm = tq.c.z > 0.0f ? tq.c.y / tq.c.z : 0.0f;
            const Surf &ps = sPrev[tqid];
            const V3 toCur = c.lpos - ld3(s.p), toPrev = c.lpos - ld3(ps.p);
            const float curD2 = fmax_ref(dot(toCur, toCur), kRayEps), prevD2 = fmax_ref(dot(toPrev, toPrev), kRayEps);
            const V3 wiCur = normalize(toCur), wiPrev = normalize(toPrev);
            const float cosCur = fmax_ref(dot(normalize(ld3(s.n)), wiCur), 0.0f);
            const float cosPrev = fmax_ref(dot(normalize(normalize(ld3(ps.n))), wiPrev), 0.0f);
            float J = (prevD2 / curD2) * (cosCur / fmax_ref(cosPrev, kRayEps));
            if (!isfinite(J) || J < 0.0f) J = 0.0f;
            else J = fmin_ref(J, 32.0f);
            float w = prevTarget > 0.0f ? norm * (target / prevTarget) * J : 0.0f;
            const float tp = fmax_ref(c.pdf, 0.0f);
            float den = tp * (currentM + totalSpatialM);
            den = den + tq.c.z * tp * J;
            const float mis = den > 0.0f ? (tq.c.z * tp * J) / den : 0.0f;
            w = w * mis;
            const U4 rr = philox(U4{pixel, sample, 0x21000u, v.index}, v.k0, v.k1);
            ref_update(r, contrib, c, cc, w, tq.c.z, u01(rr.x));
          }
        }
        if (__float_as_int(r.a.w) >= 0 && r.c.w > 0.0f && r.c.z > 0.0f) {
          const float norm = r.c.y / (r.c.z * r.c.w);
          const V3 add = contrib * norm;
          // an entry whose ray interval is empty: never occluded, resolved with the shadow rays
          A = make_float4(s.p.x, s.p.y, s.p.z, kRayEps);
          B = make_float4(0.0f, 0.0f, 1.0f, kRayEps);
          Cc = make_float4(add.x, add.y, add.z, 0.0f);
          want = true;
        }
      }
      rOut[pid] = r;
    }
    const uint32_t slot = warp_append(&cnt->qlen[kQ * (2)], want);
    if (want) {
      sRays[2 * slot] = A;
      sRays[2 * slot + 1] = B;
      sIds[slot] = (uint32_t)pid;
      sContrib[slot] = Cc;
    }
  }
}

// Reuse visibility: bit k of the path's byte-sized mask word.
__global__ void __launch_bounds__(kPtBlock) k_restir_ref_vis5(const uint32_t *__restrict__ ids,
                                                              const uint8_t *__restrict__ occ,
                                                              uint32_t *__restrict__ mask, Counters *cnt) {
  const uint32_t n = cnt->qlen[kQ * (3)];
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (occ[i]) continue;
    const uint32_t id = ids[i], pid = id / kRefReuse, k = id - pid * kRefReuse;
    atomicOr(&mask[pid], 1u << k);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt->stats[2] += n;
}

nomad_status restir_prepare(nomad_ctx *ctx, uint32_t nviews, const nomad_view *views, unsigned long long P,
                            RestirPlan &plan) {
  FrameState &F = ctx->frame;
  if (F.restirPaths < P) {
    NOMAD_CUDA(ctx, F.rInit.reserve(P * sizeof(Resv)));
    NOMAD_CUDA(ctx, F.rTemp.reserve(P * sizeof(Resv)));
    for (int k = 0; k < 2; ++k) {
      NOMAD_CUDA(ctx, F.resv[k].reserve(P * sizeof(Resv)));
      NOMAD_CUDA(ctx, F.surf[k].reserve(P * sizeof(Surf)));
    }
    F.restirPaths = P;
    F.restirValid = false;
  }
  if (F.restir.reference_mode) {
    const uint64_t per = std::max<uint64_t>(F.restir.candidates, kRefReuse);
    if (P * per >= 0xffffffffull) return nomad_fail(ctx, NOMAD_ERR_LIMIT, "too many reference-mode ReSTIR candidates");
    if (F.refRayCap < P * per) {
      NOMAD_CUDA(ctx, F.refRays.reserve(P * per * 32));
      NOMAD_CUDA(ctx, F.refIds.reserve(P * per * 4));
      NOMAD_CUDA(ctx, F.refOcc.reserve(P * per));
      F.refRayCap = P * per;
    }
    if (F.refPaths < P) {
      NOMAD_CUDA(ctx, F.refMask.reserve(P * 8));
      NOMAD_CUDA(ctx, F.reuseMask.reserve(P * 4));
      NOMAD_CUDA(ctx, F.refContrib.reserve(P * 16));
      F.refPaths = P;
    }
  }
  NOMAD_CUDA(ctx, F.prevViews.reserve(nviews * sizeof(ViewDev)));
  bool compatible = F.restirValid && F.prevHostViews.size() == nviews;
  for (uint32_t i = 0; compatible && i < nviews; ++i) {
    const nomad_view &a = views[i], &b = F.prevHostViews[i];
    compatible = a.width == b.width && a.height == b.height && a.spp == b.spp;
  }
  plan.on = true;
  plan.cur = F.restirCur;
  plan.cfg = F.restir;
  plan.temporal = (compatible && F.restir.temporal) ? 1 : 0;
  return NOMAD_OK;
}

nomad_status restir_launch(nomad_ctx *ctx, uint32_t nviews, unsigned long long P, const Lights &L, Counters *C,
                           const RestirPlan &plan) {
  FrameState &F = ctx->frame;
  cudaStream_t s = ctx->stream;
  const nomad_restir_config &cf = plan.cfg;
  RestirDev cfg{cf.candidates, cf.temporal, cf.spatial, cf.radius_px, cf.m_cap};
  const ViewDev *V = F.views.as<const ViewDev>();
  const int cur = plan.cur;
  const int grid = ctx->smCount * 8;
  Surf *sCur = F.surf[cur].as<Surf>();
  if (cf.reference_mode) {
    const RefArgs ra{F.lightPdf.as<const float>(), ctx->primCount, (cf.candidates + 31) / 32};
    const ViewDev *PV = F.prevViews.as<const ViewDev>();
    k_restir_ref_reset<<<1, 1, 0, s>>>(C);
    k_restir_ref_cand<<<grid, kPtBlock, 0, s>>>(V, nviews, P, cfg, F.qRays[0].as<const float4>(),
                                               F.hits.as<const int32_t>(),
                                               ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()}, L, sCur, F.refMask.as<uint32_t>(), ra,
                                               F.refRays.as<float4>(), F.refIds.as<uint32_t>(), C);
    NOMAD_CUDA(ctx, cudaGetLastError());
    nomad_status ts = nomad_trace_variant(ctx, ctx->trav, true, F.refRays.as<const float4>(), P * cf.candidates,
                                          &C->qlen[kQ * (3)], &C->cursor[1], nullptr, F.refOcc.as<uint8_t>(), nullptr, s);
    if (ts != NOMAD_OK) return ts;
    k_restir_ref_vis<<<grid, kPtBlock, 0, s>>>(F.refIds.as<const uint32_t>(), F.refOcc.as<const uint8_t>(),
                                              cf.candidates, ra.words, F.refMask.as<uint32_t>(), C);
    k_restir_ref_reset<<<1, 1, 0, s>>>(C);
    k_restir_ref_reuse<<<grid, kPtBlock, 0, s>>>(V, PV, nviews, P, cfg, ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()}, L, sCur,
                                                F.refMask.as<const uint32_t>(), ra, F.resv[cur ^ 1].as<const Resv>(),
                                                F.surf[cur ^ 1].as<const Surf>(), plan.temporal, F.rInit.as<Resv>(),
                                                F.refContrib.as<float4>(), F.reuseMask.as<uint32_t>(),
                                                F.refRays.as<float4>(), F.refIds.as<uint32_t>(), C);
    NOMAD_CUDA(ctx, cudaGetLastError());
    ts = nomad_trace_variant(ctx, ctx->trav, true, F.refRays.as<const float4>(), P * kRefReuse, &C->qlen[kQ * (3)],
                             &C->cursor[1], nullptr, F.refOcc.as<uint8_t>(), nullptr, s);
    if (ts != NOMAD_OK) return ts;
    k_restir_ref_vis5<<<grid, kPtBlock, 0, s>>>(F.refIds.as<const uint32_t>(), F.refOcc.as<const uint8_t>(),
                                               F.reuseMask.as<uint32_t>(), C);
    k_restir_ref_reset<<<1, 1, 0, s>>>(C);
    k_restir_ref_final<<<grid, kPtBlock, 0, s>>>(V, PV, nviews, P, ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()}, sCur, ra,
                                                F.resv[cur ^ 1].as<const Resv>(), F.surf[cur ^ 1].as<const Surf>(),
                                                plan.temporal, F.rInit.as<const Resv>(), F.refContrib.as<const float4>(),
                                                F.reuseMask.as<const uint32_t>(), F.resv[cur].as<Resv>(),
                                                F.sRays.as<float4>(), F.sIds.as<uint32_t>(), F.sContrib.as<float4>(), C);
    NOMAD_CUDA(ctx, cudaGetLastError());
    NOMAD_CUDA(ctx, cudaMemcpyAsync(F.prevViews.p, F.views.p, nviews * sizeof(ViewDev), cudaMemcpyDeviceToDevice, s));
    return NOMAD_OK;
  }
  const uint32_t cdfCap = std::min<uint32_t>(ctx->res.emissiveCount, 8192u);
  k_restir_initial<<<grid, kPtBlock, cdfCap * sizeof(float), s>>>(
      V, nviews, P, cfg, F.qRays[0].as<const float4>(), F.hits.as<const int32_t>(),
      ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()}, L, F.rInit.as<Resv>(), sCur, cdfCap);
  k_restir_temporal<<<grid, kPtBlock, 0, s>>>(V, F.prevViews.as<const ViewDev>(), nviews, P, cfg,
                                             ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()}, F.rInit.as<const Resv>(), sCur,
                                             F.resv[cur ^ 1].as<const Resv>(), F.surf[cur ^ 1].as<const Surf>(),
                                             F.rTemp.as<Resv>(), plan.temporal);
  k_restir_spatial<<<grid, kPtBlock, 0, s>>>(V, nviews, P, cfg, ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()},
                                            F.rTemp.as<const Resv>(), sCur, F.resv[cur].as<Resv>());
  k_restir_shade<<<grid, kPtBlock, 0, s>>>(V, nviews, P, ShadeTables{ctx->shadeRec.as<const float4>(), ctx->matTable.as<const float4>()}, F.resv[cur].as<const Resv>(),
                                          sCur, F.sRays.as<float4>(), F.sIds.as<uint32_t>(), F.sContrib.as<float4>(), C);
  NOMAD_CUDA(ctx, cudaGetLastError());
  NOMAD_CUDA(ctx, cudaMemcpyAsync(F.prevViews.p, F.views.p, nviews * sizeof(ViewDev), cudaMemcpyDeviceToDevice, s));
  return NOMAD_OK;
}

void restir_commit(nomad_ctx *ctx, uint32_t nviews, const nomad_view *views) {
  FrameState &F = ctx->frame;
  F.prevHostViews.assign(views, views + nviews);
  F.restirCur ^= 1;
  F.restirValid = true;
}

}  // namespace

extern "C" nomad_status nomad_set_restir(nomad_ctx *ctx, const nomad_restir_config *cfg) {
  if (!ctx || !cfg) return NOMAD_ERR_INVALID_ARGUMENT;
  if (cfg->candidates == 0 || cfg->candidates > 1024 || cfg->spatial > 16 || !(cfg->radius_px >= 0.0f) ||
      !(cfg->m_cap > 0.0f) || cfg->reference_mode > 1 || (cfg->reference_mode && cfg->candidates > 64))
    return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "ReSTIR config out of range");
  ctx->frame.restir = *cfg;
  ctx->frame.restirValid = false;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_reset_restir(nomad_ctx *ctx) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  ctx->frame.restirValid = false;
  return NOMAD_OK;
}
