// ORACLE shim — test infrastructure only. A Linux stand-in for the two pieces of Apple's
// <simd/quaternion.h> that the reference's SceneLoader.cpp uses: simd::quatf(angle, axis) and
// simd_act(q, v). Apple's implementation is not available here; this one defines the rotation
// by its textbook formula, in FP32, each operation separately rounded:
//   q = (axis * sin(angle / 2), cos(angle / 2))     (axis not renormalised)
//   simd_act(q, v) = imag(q * (v, 0) * conj(q))      (Hamilton products, left to right)
#pragma once
#include <cmath>

#include "simd.h"

namespace simd {

struct quatf {
  float ix, iy, iz, r;
  quatf() = default;
  quatf(float angle, float3 axis) {
    const float s = std::sin(angle * 0.5f), c = std::cos(angle * 0.5f);
    ix = axis.x * s;
    iy = axis.y * s;
    iz = axis.z * s;
    r = c;
  }
};

}  // namespace simd

inline simd::quatf simd_quat_mul(const simd::quatf &a, const simd::quatf &b) {
  simd::quatf o;
  o.r = a.r * b.r - a.ix * b.ix - a.iy * b.iy - a.iz * b.iz;
  o.ix = a.r * b.ix + a.ix * b.r + a.iy * b.iz - a.iz * b.iy;
  o.iy = a.r * b.iy - a.ix * b.iz + a.iy * b.r + a.iz * b.ix;
  o.iz = a.r * b.iz + a.ix * b.iy - a.iy * b.ix + a.iz * b.r;
  return o;
}

inline simd::float3 simd_act(const simd::quatf &q, simd::float3 v) {
  simd::quatf p;
  p.ix = v.x;
  p.iy = v.y;
  p.iz = v.z;
  p.r = 0.0f;
  simd::quatf c;
  c.ix = -q.ix;
  c.iy = -q.iy;
  c.iz = -q.iz;
  c.r = q.r;
  const simd::quatf o = simd_quat_mul(simd_quat_mul(q, p), c);
  return simd::make_float3(o.ix, o.iy, o.iz);
}
