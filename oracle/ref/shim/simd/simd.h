// ORACLE shim — test infrastructure only. A Linux stand-in for the parts of Apple's
// <simd/simd.h> that the reference's Scene headers and SceneBVH.cpp use, so that the
// reference's own builder compiles here unmodified. Semantics: 16-byte float3 (fourth lane
// padding), component-wise operators, dot = (x*x + y*y) + z*z, length = sqrtf(dot),
// min/max pick the first argument on ties.
#pragma once
#include <cmath>
#include <cstdint>

namespace simd {

struct float2 {
  float x, y;
  float2() = default;
  constexpr float2(float a, float b) : x(a), y(b) {}
  float &operator[](int i) { return (&x)[i]; }
  float operator[](int i) const { return (&x)[i]; }
};
struct alignas(16) float3 {
  float x, y, z;
  float3() = default;
  constexpr explicit float3(float s) : x(s), y(s), z(s) {}
  constexpr float3(float a, float b, float c) : x(a), y(b), z(c) {}
  float &operator[](int i) { return (&x)[i]; }
  float operator[](int i) const { return (&x)[i]; }
};
struct alignas(16) float4 {
  float x, y, z, w;
  float4() = default;
  constexpr float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
};
struct alignas(16) uint3 {
  uint32_t x, y, z;
};
struct alignas(16) float4x4 {
  float4 columns[4];
};

inline float2 operator-(float2 a, float2 b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator+(float2 a, float2 b) { return float2(a.x + b.x, a.y + b.y); }
inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator-(float3 a) { return float3(-a.x, -a.y, -a.z); }
inline float3 operator*(float3 a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float s, float3 a) { return float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator/(float3 a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator-(float3 a, float s) { return float3(a.x - s, a.y - s, a.z - s); }
inline float3 operator+(float3 a, float s) { return float3(a.x + s, a.y + s, a.z + s); }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 cross(float3 a, float3 b) {
  return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float length(float3 a) { return std::sqrt(dot(a, a)); }
inline float3 normalize(float3 a) { return a / length(a); }
inline float3 min(float3 a, float3 b) {
  return float3(b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y, b.z < a.z ? b.z : a.z);
}
inline float3 max(float3 a, float3 b) {
  return float3(a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y, a.z < b.z ? b.z : a.z);
}
inline float2 make_float2(float a, float b) { return float2(a, b); }
inline float3 make_float3(float s) { return float3(s); }
inline float3 make_float3(float a, float b, float c) { return float3(a, b, c); }
inline float4 make_float4(float3 v, float w) { return float4(v.x, v.y, v.z, w); }
inline float4 make_float4(float a, float b, float c, float d) { return float4(a, b, c, d); }
inline uint3 make_uint3(uint32_t a, uint32_t b, uint32_t c) { return uint3{a, b, c}; }

}  // namespace simd
