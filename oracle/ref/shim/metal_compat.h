// ORACLE shim — test infrastructure only. Just enough of the Metal Shading Language's
// vector types and built-ins for the reference's shader headers (Renderer/Shaders/*.h) to
// compile as C++17 on the host, so the reference's own traversal code runs here as a checker.
// Semantics chosen to match the scalar oracle: float arithmetic, dot = (x*x + y*y) + z*z,
// normalize(v) = v / sqrt(dot(v, v)), no fused multiply-add (-ffp-contract=off).
// Texture reads return zero and samples return one (the checked paths do not use textures).
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>

typedef unsigned int uint;
typedef unsigned char uchar;

struct float2 {
  float x, y;
  float2() = default;
  explicit float2(float s) : x(s), y(s) {}
  float2(float a, float b) : x(a), y(b) {}
  template <typename V> explicit float2(V v, decltype(v.x) * = nullptr) : x(float(v.x)), y(float(v.y)) {}
  float &operator[](int i) { return (&x)[i]; }
  float operator[](int i) const { return (&x)[i]; }
};
struct float3;
// Plain triple used for the read-only .xyz swizzle of a float3 (a member cannot have its own type).
struct float3_view {
  float x, y, z;
  operator float3() const;
};
struct float3 {
  union {
    struct { float x, y, z; };
    float2 xy;
    float3_view xyz;
  };
  float3() = default;
  explicit float3(float s) : x(s), y(s), z(s) {}
  float3(float a, float b, float c) : x(a), y(b), z(c) {}
  float &operator[](int i) { return (&x)[i]; }
  float operator[](int i) const { return (&x)[i]; }
};
inline float3_view::operator float3() const { return float3(x, y, z); }
// Plain pair used for the read-only .zw swizzle (anonymous members may not have constructors).
struct float2_view {
  float x, y;
  operator float2() const { return float2(x, y); }
};
struct float4 {
  union {
    struct { float x, y, z, w; };
    float3 xyz;
    float2 xy;
    struct { float xy_pad_[2]; float2_view zw; };
  };
  float4() = default;
  explicit float4(float s) : x(s), y(s), z(s), w(s) {}
  float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
  float4(float3 v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
};
struct int2 {
  int x, y;
  int2() = default;
  int2(int a, int b) : x(a), y(b) {}
  template <typename V> explicit int2(V v, decltype(v.x) * = nullptr) : x(int(v.x)), y(int(v.y)) {}
};
struct uint2 {
  uint x, y;
  uint2() = default;
  uint2(uint a, uint b) : x(a), y(b) {}
  template <typename V> explicit uint2(V v, decltype(v.x) * = nullptr) : x(uint(v.x)), y(uint(v.y)) {}
};
struct uint3 {
  uint x, y, z;
};
struct bool2 {
  bool x, y;
};
struct bool3 {
  bool x, y, z;
};
struct float4x4 {
  float4 columns[4];
};

inline float2 operator+(float2 a, float2 b) { return float2(a.x + b.x, a.y + b.y); }
inline float2 operator-(float2 a, float2 b) { return float2(a.x - b.x, a.y - b.y); }
inline float2 operator*(float2 a, float2 b) { return float2(a.x * b.x, a.y * b.y); }
inline float2 operator/(float2 a, float2 b) { return float2(a.x / b.x, a.y / b.y); }
inline float2 operator*(float2 a, float s) { return float2(a.x * s, a.y * s); }
inline float2 operator*(float s, float2 a) { return float2(s * a.x, s * a.y); }
inline float2 operator+(float2 a, float s) { return float2(a.x + s, a.y + s); }
inline float2 operator-(float2 a, float s) { return float2(a.x - s, a.y - s); }
inline float2 operator/(float2 a, float s) { return float2(a.x / s, a.y / s); }
inline bool2 operator>=(float2 a, float2 b) { return bool2{a.x >= b.x, a.y >= b.y}; }
inline bool2 operator<=(float2 a, float2 b) { return bool2{a.x <= b.x, a.y <= b.y}; }
inline int2 operator+(int2 a, int2 b) { return int2(a.x + b.x, a.y + b.y); }
inline uint2 operator+(uint2 a, uint2 b) { return uint2(a.x + b.x, a.y + b.y); }

inline float3 operator+(float3 a, float3 b) { return float3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline float3 operator-(float3 a, float3 b) { return float3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float3 operator*(float3 a, float3 b) { return float3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline float3 operator/(float3 a, float3 b) { return float3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline float3 operator-(float3 a) { return float3(-a.x, -a.y, -a.z); }
inline float3 operator*(float3 a, float s) { return float3(a.x * s, a.y * s, a.z * s); }
inline float3 operator*(float s, float3 a) { return float3(s * a.x, s * a.y, s * a.z); }
inline float3 operator/(float3 a, float s) { return float3(a.x / s, a.y / s, a.z / s); }
inline float3 operator+(float3 a, float s) { return float3(a.x + s, a.y + s, a.z + s); }
inline float3 operator-(float3 a, float s) { return float3(a.x - s, a.y - s, a.z - s); }
inline float3 &operator+=(float3 &a, float3 b) { a = a + b; return a; }
inline float3 &operator-=(float3 &a, float3 b) { a = a - b; return a; }
inline float3 &operator*=(float3 &a, float3 b) { a = a * b; return a; }
inline float3 &operator*=(float3 &a, float s) { a = a * s; return a; }
inline float3 &operator/=(float3 &a, float s) { a = a / s; return a; }

inline float4 operator+(float4 a, float4 b) { return float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
inline float4 operator*(float4 a, float4 b) { return float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }
inline float4 operator*(float4 a, float s) { return float4(a.x * s, a.y * s, a.z * s, a.w * s); }
inline float4 operator/(float4 a, float s) { return float4(a.x / s, a.y / s, a.z / s, a.w / s); }
inline float4 &operator+=(float4 &a, float4 b) { a = a + b; return a; }
inline float4 &operator/=(float4 &a, float s) { a = a / s; return a; }
inline float4 operator*(const float4x4 &m, float4 v) {
  float4 r(0.0f);
  const float *vv = &v.x;
  for (int c = 0; c < 4; ++c) r = r + m.columns[c] * vv[c];
  return r;
}

namespace metal {
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
inline float3 cross(float3 a, float3 b) {
  return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float sqrt(float x) { return std::sqrt(x); }
inline float length(float3 a) { return std::sqrt(dot(a, a)); }
inline float length_squared(float3 a) { return dot(a, a); }
inline float3 normalize(float3 a) { return a / std::sqrt(dot(a, a)); }
inline float abs(float x) { return std::fabs(x); }
inline float fabs(float x) { return std::fabs(x); }
inline float max(float a, float b) { return a < b ? b : a; }
inline float min(float a, float b) { return b < a ? b : a; }
inline uint max(uint a, uint b) { return a < b ? b : a; }
inline uint min(uint a, uint b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline float3 max(float3 a, float3 b) { return float3(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)); }
inline float3 min(float3 a, float3 b) { return float3(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)); }
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline float3 clamp(float3 v, float lo, float hi) {
  return float3(clamp(v.x, lo, hi), clamp(v.y, lo, hi), clamp(v.z, lo, hi));
}
inline float3 mix(float3 a, float3 b, float t) { return a + (b - a) * t; }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float cos(float a) { return std::cos(a); }
inline float sin(float a) { return std::sin(a); }
inline float atan2(float a, float b) { return std::atan2(a, b); }
inline float asin(float a) { return std::asin(a); }
inline float floor(float a) { return std::floor(a); }
inline float fract(float a) { return a - std::floor(a); }
inline bool isfinite(float a) { return std::isfinite(a); }
inline bool3 isfinite(float3 v) { return bool3{std::isfinite(v.x), std::isfinite(v.y), std::isfinite(v.z)}; }
inline bool all(bool3 b) { return b.x && b.y && b.z; }
inline bool all(bool2 b) { return b.x && b.y; }
inline float3 reflect(float3 i, float3 n) { return i - n * (2.0f * dot(n, i)); }
inline float3 refract(float3 i, float3 n, float eta) {
  float d = dot(n, i);
  float k = 1.0f - eta * eta * (1.0f - d * d);
  if (k < 0.0f) return float3(0.0f);
  return i * eta - n * (eta * d + std::sqrt(k));
}
template <typename T> inline T as_type(float f) {
  T t;
  std::memcpy(&t, &f, sizeof(T));
  return t;
}

namespace access { enum Mode { sample, read, write, read_write }; }
namespace address { enum Mode { repeat, clamp_to_edge }; }
namespace filter { enum Mode { nearest, linear }; }
struct sampler {
  constexpr sampler() {}
  constexpr sampler(address::Mode, filter::Mode) {}
};
struct level {
  float l;
  explicit level(float v) : l(v) {}
};
template <typename T, access::Mode M = access::sample> struct texture2d {
  float4 *data = nullptr;
  uint w = 0, h = 0;
  uint get_width() const { return w; }
  uint get_height() const { return h; }
  float4 read(uint2 p) const { return (data && p.x < w && p.y < h) ? data[p.y * w + p.x] : float4(0.0f); }
  void write(float4 v, uint2 p) const {
    if (data && p.x < w && p.y < h) data[p.y * w + p.x] = v;
  }
  float4 sample(sampler, float2) const { return float4(1.0f); }
  float4 sample(sampler, float2, level) const { return float4(1.0f); }
};
template <typename T, unsigned N> struct array {
  T items[N];
  const T &operator[](unsigned i) const { return items[i]; }
  T &operator[](unsigned i) { return items[i]; }
};
typedef std::atomic<uint32_t> atomic_uint;
const std::memory_order memory_order_relaxed = std::memory_order_relaxed;
inline uint32_t atomic_fetch_add_explicit(atomic_uint *a, uint32_t v, std::memory_order o) {
  return a->fetch_add(v, o);
}
}  // namespace metal

namespace simd {
using ::float2;
using ::float3;
using ::float4;
using ::float4x4;
}  // namespace simd

// MSL address-space qualifiers have no meaning on the host.
#define thread
#define device
#define constant const
