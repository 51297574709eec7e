// Host-side float3 helpers for the scene builder and generators.
//
// Every operation is written out in a fixed order with no fused multiply-add (this file is
// compiled with -ffp-contract=off), so the packed scene arrays are bit-reproducible:
// dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z, cross is the textbook determinant, and
// length = sqrtf(dot(v,v)).
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>

// Host and device (the GPU scene packer uses the same operations).
#ifdef __CUDACC__
#define NOMAD_HD __host__ __device__
#else
#define NOMAD_HD
#endif

namespace nomad {

struct V3 {
  float x, y, z;
  NOMAD_HD V3() : x(0), y(0), z(0) {}
  NOMAD_HD V3(float a, float b, float c) : x(a), y(b), z(c) {}
  NOMAD_HD explicit V3(float s) : x(s), y(s), z(s) {}
  NOMAD_HD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};

NOMAD_HD inline V3 operator+(V3 a, V3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
NOMAD_HD inline V3 operator-(V3 a, V3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
NOMAD_HD inline V3 operator-(V3 a) { return V3(-a.x, -a.y, -a.z); }
NOMAD_HD inline V3 operator*(V3 a, float s) { return V3(a.x * s, a.y * s, a.z * s); }
NOMAD_HD inline V3 operator*(float s, V3 a) { return V3(s * a.x, s * a.y, s * a.z); }
NOMAD_HD inline V3 operator/(V3 a, float s) { return V3(a.x / s, a.y / s, a.z / s); }
NOMAD_HD inline V3 operator-(V3 a, float s) { return V3(a.x - s, a.y - s, a.z - s); }
NOMAD_HD inline V3 operator+(V3 a, float s) { return V3(a.x + s, a.y + s, a.z + s); }
NOMAD_HD inline float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
NOMAD_HD inline V3 cross(V3 a, V3 b) {
  return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
NOMAD_HD inline float length(V3 a) { return std::sqrt(dot(a, a)); }
NOMAD_HD inline V3 vmin(V3 a, V3 b) {
  return V3(b.x < a.x ? b.x : a.x, b.y < a.y ? b.y : a.y, b.z < a.z ? b.z : a.z);
}
NOMAD_HD inline V3 vmax(V3 a, V3 b) {
  return V3(a.x < b.x ? b.x : a.x, a.y < b.y ? b.y : a.y, a.z < b.z ? b.z : a.z);
}
NOMAD_HD inline bool finite3(V3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }

NOMAD_HD inline float int_bits_as_float(int32_t i) {
  float f;
  std::memcpy(&f, &i, 4);
  return f;
}
NOMAD_HD inline int32_t float_bits_as_int(float f) {
  int32_t i;
  std::memcpy(&i, &f, 4);
  return i;
}

}  // namespace nomad
