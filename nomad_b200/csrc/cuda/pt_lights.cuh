// Emissive primitives for next-event estimation and ReSTIR.
//
// light_shape() computes what does not depend on the sample (vertices or centre and edges, unit
// normal, area); light_point() places a sample on it. The path tracer's light sampling
// (sampleLightPoint, PathTracing.h:582-643) and the per-frame light records below both call
// these, so a record holds exactly the values the per-sample code would compute.
#pragma once
#include "pt_math.cuh"

namespace nomad_pt {

constexpr float kLightPi = 3.14159265358979323846f;

struct LightShape {
  int type;     // 0 sphere, 1 triangle, 2 rectangle
  V3 a, b, c;   // triangle v0 v1 v2; rectangle centre, edge u, edge v; sphere centre, (radius, ., .)
  V3 nrm;       // unit normal (triangle, rectangle)
  float area;
  bool valid;   // the sampler would accept this primitive
};

__device__ __forceinline__ LightShape light_shape(const float4 *__restrict__ prims, uint32_t lp) {
  const float4 *g = prims + 7ll * lp;
  const float4 p0 = __ldg(g), p1 = __ldg(g + 1), p2 = __ldg(g + 2);
  LightShape s;
  s.type = (int)p0.w;
  s.a = ld3(p0);
  s.b = ld3(p1);
  s.c = ld3(p2);
  s.nrm = v3(0.0f, 0.0f, 0.0f);
  s.area = 0.0f;
  s.valid = false;
  if (s.type == 0) {
    const float radius = p1.x;
    if (radius <= 0.0f) return s;
    s.area = 4.0f * kLightPi * radius * radius;
  } else if (s.type == 1) {
    const V3 n = cross(s.b - s.a, s.c - s.a);
    const float ln = length(n);
    if (ln <= 0.0f) return s;
    s.nrm = n / ln;
    s.area = 0.5f * ln;
  } else if (s.type == 2) {
    const V3 n = cross(s.b, s.c);
    const float ln = length(n);
    if (ln <= 0.0f) return s;
    s.nrm = n / ln;
    s.area = 4.0f * ln;
  } else {
    return s;
  }
  s.valid = s.area > 0.0f;
  return s;
}

// Sample position on the shape for (u1, u2); `nrm` receives the normal there.
__device__ __forceinline__ V3 light_point(const LightShape &s, float u1, float u2, V3 &nrm) {
  if (s.type == 0) {
    const float z = 2.0f * u1 - 1.0f;
    float sn, cs;
    sincos_turns(u2, sn, cs);
    const float r = sqrtf(fmax_ref(0.0f, 1.0f - z * z));
    const V3 dir = v3(r * cs, r * sn, z);
    nrm = dir;
    return s.a + dir * s.b.x;
  }
  nrm = s.nrm;
  if (s.type == 1) {
    const float su1 = sqrtf(u1);
    const float b0 = 1.0f - su1, b1 = su1 * (1.0f - u2), b2 = su1 * u2;
    return s.a * b0 + s.b * b1 + s.c * b2;
  }
  const float su = u1 * 2.0f - 1.0f, sv = u2 * 2.0f - 1.0f;
  return s.a + s.b * su + s.c * sv;
}

// Per-frame light record of CDF slot k (5 float4): shape, normal and prim, the light-selection
// pdf and 1/area (as the samplers compute them), the ReSTIR candidate pdf constant, radiance.
//   [0] a.xyz, lpdf = weight / total      [1] b.xyz, 1 / area
//   [2] c.xyz, q = lpdf * (1 / area)      [3] nrm.xyz, prim
//   [4] emission * power, type + 1 when the sampler accepts the primitive, else 0
__device__ __forceinline__ void light_record(const float4 *__restrict__ prims, const float4 *__restrict__ mats,
                                             uint32_t lp, float wgt, float total, float4 *__restrict__ rec) {
  const LightShape s = light_shape(prims, lp);
  const float lpdf = wgt > 0.0f ? wgt / total : 0.0f;
  const float inv = s.valid ? 1.0f / s.area : 0.0f;
  const float q = lpdf * inv;
  const float4 m2 = __ldg(mats + 5ll * lp + 2);
  const V3 emission = vmax0(ld3(m2));
  const float power = fmax_ref(m2.w, 0.0f);
  const V3 lrad = emission * power;
  rec[0] = make_float4(s.a.x, s.a.y, s.a.z, lpdf);
  rec[1] = make_float4(s.b.x, s.b.y, s.b.z, inv);
  rec[2] = make_float4(s.c.x, s.c.y, s.c.z, q);
  rec[3] = make_float4(s.nrm.x, s.nrm.y, s.nrm.z, __int_as_float((int32_t)lp));
  rec[4] = make_float4(lrad.x, lrad.y, lrad.z, s.valid ? (float)(s.type + 1) : 0.0f);
}

// Shape of a record whose [4].w is positive (the sampler accepts it); area is not restored.
__device__ __forceinline__ LightShape record_shape(const float4 *__restrict__ rec) {
  const float4 r0 = __ldg(rec), r1 = __ldg(rec + 1), r2 = __ldg(rec + 2), r3 = __ldg(rec + 3), r4 = __ldg(rec + 4);
  LightShape s;
  s.type = (int)r4.w - 1;
  s.a = ld3(r0);
  s.b = ld3(r1);
  s.c = ld3(r2);
  s.nrm = ld3(r3);
  s.area = 0.0f;
  s.valid = true;
  return s;
}

}  // namespace nomad_pt
