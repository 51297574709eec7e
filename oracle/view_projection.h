// ORACLE — test infrastructure only. The previous-frame view-projection matrix that the shading
// pin hands the reference's rayColor (oracle/ref/ref_shade.cpp), and the reference's arithmetic
// on it (PathTracing.h:1433-1445), so the contract oracle can reproject exactly as the reference
// does when it runs under the reference's rules.
//
// The matrix maps a point p to NDC whose x, y give the uv in [0, 1]^2 of the pinhole view's pixel
// grid (rows from the top, as the raygen numbers them: viewportV points down). The camera maps p
// to the point where the ray from the camera C through p meets the image plane through the first
// pixel position F spanned by U and V; u = dot(q - F, U) / |U|^2 is a ratio of two affine functions
// of p, so the map is projective. Rows: x = (2u - 1) w, y = (2v - 1) w, z = 0, w = dot(p - C, U x V)
// with its sign chosen positive in front of the camera. Built in double, stored as float,
// column-major (columns[c][row]).
#pragma once
#include <cstdint>

namespace oracle_vp {

inline void build(const float cam[3], const float vu[3], const float vv[3], const float fp[3], float out[16]) {
  double C[3], U[3], V[3], F[3];
  for (int k = 0; k < 3; ++k) C[k] = cam[k], U[k] = vu[k], V[k] = vv[k], F[k] = fp[k];
  auto dot = [](const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
  const double pn[3] = {U[1] * V[2] - U[2] * V[1], U[2] * V[0] - U[0] * V[2], U[0] * V[1] - U[1] * V[0]};
  const double FC[3] = {F[0] - C[0], F[1] - C[1], F[2] - C[2]}, CF[3] = {-FC[0], -FC[1], -FC[2]};
  const double num = dot(FC, pn);
  const double sgn = num < 0 ? -1.0 : 1.0;
  // W(p) = dot(p, pn) - dot(C, pn); X(p) = (dot(C - F, A) W(p) + num (dot(p, A) - dot(C, A))) / |A|^2
  const double rowW[4] = {pn[0], pn[1], pn[2], -dot(C, pn)};
  double rows[2][4];
  const double *axes[2] = {U, V};
  for (int a = 0; a < 2; ++a) {
    const double *A = axes[a];
    const double aa = dot(A, A), cfa = dot(CF, A);
    for (int k = 0; k < 3; ++k) rows[a][k] = (cfa * pn[k] + num * A[k]) / aa;
    rows[a][3] = (cfa * rowW[3] - num * dot(C, A)) / aa;
    for (int k = 0; k < 4; ++k) rows[a][k] = 2.0 * rows[a][k] - rowW[k];
  }
  for (int c = 0; c < 4; ++c) {
    out[4 * c + 0] = (float)(sgn * rows[0][c]);
    out[4 * c + 1] = (float)(sgn * rows[1][c]);
    out[4 * c + 2] = 0.0f;
    out[4 * c + 3] = (float)(sgn * rowW[c]);
  }
}

// The reference's reprojection of p through matrix m into a w x h grid (PathTracing.h:1433-1445,
// float4x4 * float4 summed column by column as the shim does). False when p falls outside.
inline bool reproject(const float m[16], const float p[3], uint32_t w, uint32_t h, uint32_t &px, uint32_t &py) {
  float r[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  const float v[4] = {p[0], p[1], p[2], 1.0f};
  for (int c = 0; c < 4; ++c)
    for (int k = 0; k < 4; ++k) r[k] = r[k] + m[4 * c + k] * v[c];
  if (!(r[3] > 1e-4f)) return false;
  const float nx = r[0] / r[3], ny = r[1] / r[3];
  const float ux = nx * 0.5f + 0.5f, uy = ny * 0.5f + 0.5f;
  if (!(ux >= 0.0f && uy >= 0.0f && ux <= 1.0f && uy <= 1.0f)) return false;
  if (w == 0 || h == 0) return false;
  px = (uint32_t)(ux * (float)w);
  py = (uint32_t)(uy * (float)h);
  if (px > w - 1) px = w - 1;
  if (py > h - 1) py = h - 1;
  return true;
}

}  // namespace oracle_vp
