// Device math for the wavefront path tracer.
//
// Everything here is built from IEEE basic operations (+ - * /, sqrt) only, compiled with
// -fmad=false, so a host restatement with the same operation order rounds identically:
//   * Philox4x32-10 counter-based RNG (Salmon, Moraes, Dror, Shaw, "Parallel random numbers:
//     as easy as 1, 2, 3", SC'11), implemented from the paper's round function and constants;
//   * sin/cos of 2*pi*u by octant reduction and Taylor polynomials (coefficients 1/n!);
//   * log2/exp2 (for the specular lobe exponent) by exponent extraction plus series:
//     ln(m) = 2 atanh((m-1)/(m+1)) and 2^f = e^(f ln 2) by Taylor series.
#pragma once
#include <cstdint>

namespace nomad_pt {

struct V3 {
  float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 ld3(const float4 &f) { return V3{f.x, f.y, f.z}; }
__device__ __forceinline__ V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float length(V3 a) { return sqrtf(dot(a, a)); }
__device__ __forceinline__ V3 normalize(V3 a) {
  float l = sqrtf(dot(a, a));
  return a / l;
}
__device__ __forceinline__ bool finite3(V3 a) { return isfinite(a.x) && isfinite(a.y) && isfinite(a.z); }
__device__ __forceinline__ float fmax_ref(float a, float b) { return a < b ? b : a; }
__device__ __forceinline__ float fmin_ref(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ float clamp01(float x) { return fmin_ref(fmax_ref(x, 0.0f), 1.0f); }
__device__ __forceinline__ V3 vmax0(V3 a) { return v3(fmax_ref(a.x, 0.0f), fmax_ref(a.y, 0.0f), fmax_ref(a.z, 0.0f)); }
__device__ __forceinline__ float luminance(V3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }
__device__ __forceinline__ V3 reflect(V3 i, V3 n) { return i - n * (2.0f * dot(n, i)); }
__device__ __forceinline__ float pow5(float x) {
  float x2 = x * x;
  return x2 * x2 * x;
}

// ---- Philox4x32-10 ----
struct U4 {
  uint32_t x, y, z, w;
};
__device__ __forceinline__ U4 philox(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
    k0 += W0;
    k1 += W1;
  }
  return c;
}
// 24-bit uniform in [0, 1).
__device__ __forceinline__ float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

// ---- sin/cos(2*pi*u), u in [0, 1) ----
__device__ __forceinline__ void sincos_turns(float u, float &s, float &c) {
  // octant reduction on the turn fraction: u*8 = o + f, angle = (f - 0.5) * pi/4 around the
  // octant centre (|x| <= pi/8).
  float t = u * 8.0f;
  float fo = floorf(t);
  int o = (int)fo & 7;
  float x = (t - fo - 0.5f) * 0.785398163397448f;  // pi / 4
  float x2 = x * x;
  float sx = x * (1.0f - x2 * (0.16666666666666667f - x2 * (0.008333333333333333f - x2 * 0.0001984126984126984f)));
  float cx = 1.0f - x2 * (0.5f - x2 * (0.041666666666666667f - x2 * (0.001388888888888889f - x2 * 2.48015873015873e-05f)));
  // angle = (o + 0.5) * pi/4 + x; rotate (cx, sx) by the octant centre.
  const float kc[8] = {0.923879532511287f, 0.382683432365090f, -0.382683432365090f, -0.923879532511287f,
                       -0.923879532511287f, -0.382683432365090f, 0.382683432365090f, 0.923879532511287f};
  const float ks[8] = {0.382683432365090f, 0.923879532511287f, 0.923879532511287f, 0.382683432365090f,
                       -0.382683432365090f, -0.923879532511287f, -0.923879532511287f, -0.382683432365090f};
  float cc = kc[o], ss = ks[o];
  c = cc * cx - ss * sx;
  s = ss * cx + cc * sx;
}

// ---- log2 / exp2 ----
__device__ __forceinline__ float log2_series(float a) {
  // a > 0, finite. a = m * 2^e with m in [sqrt(1/2), sqrt(2)).
  int e;
  float m = frexpf(a, &e);  // m in [0.5, 1)
  if (m < 0.70710678118654752f) {
    m = m * 2.0f;
    e -= 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float ln = 2.0f * s * (1.0f + s2 * (0.3333333333333333f + s2 * (0.2f + s2 * (0.14285714285714285f + s2 * 0.1111111111111111f))));
  return (float)e + ln * 1.4426950408889634f;  // 1 / ln 2
}
__device__ __forceinline__ float exp2_series(float y) {
  if (y < -126.0f) return 0.0f;
  if (y > 127.0f) return INFINITY;
  float fi = floorf(y);
  float f = (y - fi) * 0.6931471805599453f;  // ln 2, f in [0, ln 2)
  float p = 1.0f + f * (1.0f + f * (0.5f + f * (0.16666666666666667f + f * (0.041666666666666667f +
            f * (0.008333333333333333f + f * (0.001388888888888889f + f * (0.0001984126984126984f +
            f * 2.48015873015873e-05f)))))));
  return ldexpf(p, (int)fi);
}
// a^b for a in (0, 1], b > 0 (the specular lobe's cosTheta = u^(1/(n+1))).
__device__ __forceinline__ float pow_pos(float a, float b) {
  if (!(a > 0.0f)) return 0.0f;
  return exp2_series(b * log2_series(a));
}

}  // namespace nomad_pt
