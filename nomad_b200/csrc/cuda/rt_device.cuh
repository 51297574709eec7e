// Device-side traversal over the pair-node layout (see host/layout.h).
//
// Semantics restated from the reference's firstHitTLAS / firstHitBVH / intersectAABB
// (Nomad Path Tracer/Renderer/Shaders/PathTracing.h:646-1066):
//   * box test: slab test over [RAY_EPS, bound]; an axis with |d| < RAY_EPS is "parallel" and
//     only requires the origin to lie inside that slab (:648-654); a box is missed when
//     tMax < tMin (:663);
//   * triangle test: Möller–Trumbore with |a| > 1e-5, u in [0,1], v >= 0, u+v <= 1,
//     accepted when RAY_EPS < t < best (:786-797);
//   * rectangle (:849-913) and sphere (:751-770) tests as in the reference;
//   * primitives marked inactive are skipped (:723); non-resident instances are skipped (:1006).
// Differences that make the result independent of traversal order (so every kernel variant
// returns the same hit as the scalar oracle):
//   * ties in t go to the lowest primitive index (the reference keeps the first found);
//   * boxes are pruned against best_t * (1 + 2^-10) instead of best_t, so a box whose entry
//     distance rounds a few ulps past an equal-t hit is still visited;
//   * no silent stack-overflow drop: the host sizes the stack from the tree depth, and a guard
//     sets a status bit instead of dropping work unnoticed.
// This translation unit is compiled with -fmad=false, and every expression below is written in
// the operation order the oracle uses, so t, u and v are bit-identical to the oracle's.
#pragma once
#include <cstdint>

namespace nomad_dev {

constexpr float kRayEps = 1e-4f;
// One-sample NEE: a light counts as visible when the closest hit is the light itself no nearer
// than dist - 0.001 (PathTracing.h:1832-1834), so the shadow ray's any-hit window ends there.
constexpr float kNeeShadowEps = 0.001f;
constexpr float kPruneScale = 1.0009765625f;  // 1 + 2^-10
constexpr int32_t kEmptyRef = INT32_MIN;
constexpr int32_t kLastInLeaf = 1 << 8;
constexpr uint32_t kStatusStackOverflow = 1u << 0;

struct DevScene {
  const float4 *__restrict__ pn;     // pair nodes, 4 float4 each
  const float4 *__restrict__ tri;    // leaf-ordered triangle records, 3 float4 each
  const float4 *__restrict__ prims;  // SceneBVH packed primitives, 7 float4 each
  float rmin[3], rmax[3];
  int32_t rootRef;
  uint32_t tlasPairs;
  uint32_t *status;
};

struct RayP {
  float ox, oy, oz, dx, dy, dz, ix, iy, iz;
  int par;  // bit i set: axis i treated as parallel
};

__device__ __forceinline__ float4 ldg4(const float4 *p) { return __ldg(p); }

__device__ __forceinline__ RayP prep_ray(float4 a, float4 b) {
  RayP r;
  r.ox = a.x; r.oy = a.y; r.oz = a.z;
  r.dx = b.x; r.dy = b.y; r.dz = b.z;
  r.par = (fabsf(b.x) < kRayEps ? 1 : 0) | (fabsf(b.y) < kRayEps ? 2 : 0) |
          (fabsf(b.z) < kRayEps ? 4 : 0);
  // 1.0 / dir, correctly rounded, as intersectAABB computes it per axis (:655).
  r.ix = __frcp_rn(b.x);
  r.iy = __frcp_rn(b.y);
  r.iz = __frcp_rn(b.z);
  return r;
}

// intersectAABB over [kRayEps, bound]; returns the entry distance in tnear.
__device__ __forceinline__ bool slab(const RayP &r, float mnx, float mny, float mnz, float mxx,
                                     float mxy, float mxz, float bound, float &tnear) {
  float tn = kRayEps, tf = bound;
  if (r.par == 0) {
    float t0 = (mnx - r.ox) * r.ix, t1 = (mxx - r.ox) * r.ix;
    float u0 = (mny - r.oy) * r.iy, u1 = (mxy - r.oy) * r.iy;
    float w0 = (mnz - r.oz) * r.iz, w1 = (mxz - r.oz) * r.iz;
    tn = fmaxf(fmaxf(fminf(t0, t1), fminf(u0, u1)), fmaxf(fminf(w0, w1), tn));
    tf = fminf(fminf(fmaxf(t0, t1), fmaxf(u0, u1)), fminf(fmaxf(w0, w1), tf));
  } else {
    bool ok = true;
    if (r.par & 1) {
      ok = ok && !(r.ox < mnx || r.ox > mxx);
    } else {
      float t0 = (mnx - r.ox) * r.ix, t1 = (mxx - r.ox) * r.ix;
      tn = fmaxf(tn, fminf(t0, t1));
      tf = fminf(tf, fmaxf(t0, t1));
    }
    if (r.par & 2) {
      ok = ok && !(r.oy < mny || r.oy > mxy);
    } else {
      float t0 = (mny - r.oy) * r.iy, t1 = (mxy - r.oy) * r.iy;
      tn = fmaxf(tn, fminf(t0, t1));
      tf = fminf(tf, fmaxf(t0, t1));
    }
    if (r.par & 4) {
      ok = ok && !(r.oz < mnz || r.oz > mxz);
    } else {
      float t0 = (mnz - r.oz) * r.iz, t1 = (mxz - r.oz) * r.iz;
      tn = fmaxf(tn, fminf(t0, t1));
      tf = fminf(tf, fmaxf(t0, t1));
    }
    if (!ok) {
      tnear = tn;
      return false;
    }
  }
  tnear = tn;
  return !(tf < tn);
}

struct HitRec {
  float t, u, v;
  int32_t prim, inst;
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
  return ax * bx + ay * by + az * bz;
}

// Tests one record; on acceptance updates h (closest) and returns true.
// `best`/`bprim` define the current closest; for any-hit `best` is tmax and bprim INT_MIN.
__device__ __forceinline__ bool test_prim(const DevScene &S, const RayP &r, float4 A, float4 B,
                                          float4 C, int32_t pid, int type, HitRec &h) {
  float tt, u = 0.0f, v = 0.0f;
  if (type == 1) {
    // Möller–Trumbore (PathTracing.h:786-797) on v0 = A, edge1 = B, edge2 = C.
    float hx = r.dy * C.z - r.dz * C.y;
    float hy = r.dz * C.x - r.dx * C.z;
    float hz = r.dx * C.y - r.dy * C.x;
    float a = dot3(B.x, B.y, B.z, hx, hy, hz);
    if (!(fabsf(a) > 1e-5f)) return false;
    float f = __frcp_rn(a);
    float sx = r.ox - A.x, sy = r.oy - A.y, sz = r.oz - A.z;
    u = f * dot3(sx, sy, sz, hx, hy, hz);
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    float qx = sy * B.z - sz * B.y;
    float qy = sz * B.x - sx * B.z;
    float qz = sx * B.y - sy * B.x;
    v = f * dot3(r.dx, r.dy, r.dz, qx, qy, qz);
    if (!(v >= 0.0f && u + v <= 1.0f)) return false;
    tt = f * dot3(C.x, C.y, C.z, qx, qy, qz);
  } else if (type == 2) {
    // Rectangle (PathTracing.h:849-872): center A, e1 B, e2 C; stored normal in prims[6].
    float fx = B.y * C.z - B.z * C.y, fy = B.z * C.x - B.x * C.z, fz = B.x * C.y - B.y * C.x;
    float fl = dot3(fx, fy, fz, fx, fy, fz);
    bool ffin = isfinite(fx) && isfinite(fy) && isfinite(fz);
    float nx, ny, nz;
    if (fl > kRayEps && ffin) {
      float len = sqrtf(fl);
      nx = fx / len; ny = fy / len; nz = fz / len;
    } else {
      nx = 0.0f; ny = 1.0f; nz = 0.0f;
    }
    float4 sn = ldg4(S.prims + 7ll * pid + 6);
    float nl = dot3(sn.x, sn.y, sn.z, sn.x, sn.y, sn.z);
    if (nl > kRayEps && isfinite(sn.x) && isfinite(sn.y) && isfinite(sn.z)) {
      float len = sqrtf(nl);
      nx = sn.x / len; ny = sn.y / len; nz = sn.z / len;
    }
    float denom = dot3(nx, ny, nz, r.dx, r.dy, r.dz);
    if (!(fabsf(denom) > 1e-5f)) return false;
    tt = dot3(A.x - r.ox, A.y - r.oy, A.z - r.oz, nx, ny, nz) / denom;
    if (!(tt > kRayEps && tt <= h.t)) return false;
    float px = r.ox + tt * r.dx, py = r.oy + tt * r.dy, pz = r.oz + tt * r.dz;
    float rx = px - A.x, ry = py - A.y, rz = pz - A.z;
    float uu = dot3(rx, ry, rz, B.x, B.y, B.z) / dot3(B.x, B.y, B.z, B.x, B.y, B.z);
    float vv = dot3(rx, ry, rz, C.x, C.y, C.z) / dot3(C.x, C.y, C.z, C.x, C.y, C.z);
    if (!(fabsf(uu) <= 1.0f && fabsf(vv) <= 1.0f)) return false;
  } else if (type == 0) {
    // Sphere (PathTracing.h:751-770): center A, radius B.x; nearest root only.
    float ocx = r.ox - A.x, ocy = r.oy - A.y, ocz = r.oz - A.z;
    float a = dot3(r.dx, r.dy, r.dz, r.dx, r.dy, r.dz);
    float b = dot3(ocx, ocy, ocz, r.dx, r.dy, r.dz);
    float c = dot3(ocx, ocy, ocz, ocx, ocy, ocz) - B.x * B.x;
    float disc = b * b - a * c;
    if (!(disc > 0.0f)) return false;
    tt = (-b - sqrtf(disc)) / a;
  } else {
    return false;
  }
  if (!(tt > kRayEps)) return false;
  if (!(tt < h.t || (tt == h.t && pid < h.prim))) return false;
  h.t = tt;
  h.u = u;
  h.v = v;
  h.prim = pid;
  h.inst = __float_as_int(B.w);
  return true;
}

struct Work {
  uint32_t nodes, tests, insts;
};

// Tests the records of one leaf, from `k` to the one flagged kLastInLeaf. Returns true when an
// any-hit query found an occluder.
template <bool ANY, bool WORK>
__device__ __forceinline__ bool leaf_walk(const DevScene &S, const RayP &r, int64_t k, HitRec &h, Work &w) {
  for (;;) {
    const float4 *q = S.tri + 3 * k;
    const float4 A = ldg4(q), B = ldg4(q + 1), C = ldg4(q + 2);
    const int32_t pid = __float_as_int(A.w);
    const int32_t meta = __float_as_int(C.w);
    if (WORK) w.tests += 1;
    if (pid >= 0 && test_prim(S, r, A, B, C, pid, meta & 0xff, h) && ANY) return true;
    if (meta & kLastInLeaf) return false;
    ++k;
  }
}

// One ray through the combined TLAS+BLAS pair-node tree.
// ANY: stop at the first accepted primitive, bound fixed at tmax.
// WORK: count box tests, primitive tests and instance-record reads.
template <int STACK, bool ANY, bool WORK>
__device__ __forceinline__ void traverse(const DevScene &S, const RayP &r, float tmax, HitRec &h,
                                         Work &w) {
  h.t = tmax;
  h.u = h.v = 0.0f;
  h.prim = ANY ? INT32_MIN : INT32_MIN;
  h.inst = -1;
  if (!(tmax > kRayEps)) {
    h.prim = -1;
    return;
  }
  float tn0;
  float bound0 = ANY ? tmax : tmax * kPruneScale;
  if (WORK) w.nodes += 1;
  if (!slab(r, S.rmin[0], S.rmin[1], S.rmin[2], S.rmax[0], S.rmax[1], S.rmax[2], bound0, tn0)) {
    h.prim = -1;
    return;
  }
  if (WORK && S.tlasPairs == 0) w.insts += 1;
  int32_t ref = S.rootRef;
  int32_t stack[STACK];
  int sp = 0;
  bool done = (ref == kEmptyRef);
  while (!done) {
    if (ref >= 0) {
      const float4 *p = S.pn + 4ll * ref;
      float4 a = ldg4(p), b = ldg4(p + 1), c = ldg4(p + 2), d = ldg4(p + 3);
      int32_t lref = __float_as_int(a.w), rref = __float_as_int(b.w);
      float bound = ANY ? tmax : h.t * kPruneScale;
      float tl, tr;
      bool hl = slab(r, a.x, a.y, a.z, b.x, b.y, b.z, bound, tl);
      bool hr = slab(r, c.x, c.y, c.z, d.x, d.y, d.z, bound, tr);
      if (WORK) {
        w.nodes += 2;
        if ((uint32_t)ref < S.tlasPairs) {
          if (hl && !(lref >= 0 && (uint32_t)lref < S.tlasPairs)) w.insts += 1;
          if (hr && !(rref >= 0 && (uint32_t)rref < S.tlasPairs)) w.insts += 1;
        }
      }
      hl = hl && lref != kEmptyRef;
      hr = hr && rref != kEmptyRef;
      if (hl && hr) {
        bool lf = !(tr < tl);
        if (sp < STACK) {
          stack[sp++] = lf ? rref : lref;
        } else {
          atomicOr(S.status, kStatusStackOverflow);
        }
        ref = lf ? lref : rref;
      } else if (hl) {
        ref = lref;
      } else if (hr) {
        ref = rref;
      } else {
        if (sp == 0) break;
        ref = stack[--sp];
      }
      continue;
    }
    // Leaf: records ~ref .. up to the one flagged kLastInLeaf.
    if (leaf_walk<ANY, WORK>(S, r, ~(int64_t)ref, h, w)) done = true;
    if (done || sp == 0) break;
    ref = stack[--sp];
  }
  if (h.prim == INT32_MIN) {
    h.prim = -1;
    h.inst = -1;
  }
}

}  // namespace nomad_dev
