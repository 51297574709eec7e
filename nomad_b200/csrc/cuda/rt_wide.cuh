// Wide (4- and 8-child) traversal over the layout built by host/wide.cpp.
//
// Same contract as the pair-node walk in rt_device.cuh (box test, primitive tests, tie rule,
// pruning margin): a wide node's child boxes are boxes of the binary tree, so the primitives a
// ray reaches are the same and the hits are bit-identical. Per node, the W child boxes are tested
// from one structure-of-arrays fetch (7 or 14 float4 loads), the hit children are ordered by entry
// distance with a sorting network in registers, the nearest is visited next and the others are
// pushed far-to-near with their entry distance, so a popped entry that now lies beyond the
// current best hit is dropped without a fetch (its box would fail the test again).
#pragma once
#include "rt_device.cuh"

namespace nomad_dev {

struct WideScene {
  const float4 *__restrict__ wn;  // W == 4: 8 float4 per node; W == 8: 16 float4 per node
  int32_t root;
};

__device__ __forceinline__ void cswap(float &ta, int32_t &ra, float &tb, int32_t &rb) {
  if (tb < ta) {
    float t = ta;
    ta = tb;
    tb = t;
    int32_t r = ra;
    ra = rb;
    rb = r;
  }
}

template <int W>
__device__ __forceinline__ void sort_children(float (&t)[W], int32_t (&c)[W]) {
  static_assert(W == 2 || W == 4 || W == 8, "sorting networks exist for 2, 4 and 8 children");
  if constexpr (W == 2) {
    cswap(t[0], c[0], t[1], c[1]);
  } else if constexpr (W == 4) {
    cswap(t[0], c[0], t[1], c[1]);
    cswap(t[2], c[2], t[3], c[3]);
    cswap(t[0], c[0], t[2], c[2]);
    cswap(t[1], c[1], t[3], c[3]);
    cswap(t[1], c[1], t[2], c[2]);
  } else {
    // Batcher odd-even merge sort network for 8 elements (19 comparators).
#define NOMAD_CS(a, b) cswap(t[a], c[a], t[b], c[b])
    NOMAD_CS(0, 1); NOMAD_CS(2, 3); NOMAD_CS(4, 5); NOMAD_CS(6, 7);
    NOMAD_CS(0, 2); NOMAD_CS(1, 3); NOMAD_CS(4, 6); NOMAD_CS(5, 7);
    NOMAD_CS(1, 2); NOMAD_CS(5, 6);
    NOMAD_CS(0, 4); NOMAD_CS(1, 5); NOMAD_CS(2, 6); NOMAD_CS(3, 7);
    NOMAD_CS(2, 4); NOMAD_CS(3, 5);
    NOMAD_CS(1, 2); NOMAD_CS(3, 4); NOMAD_CS(5, 6);
#undef NOMAD_CS
  }
}

template <int W, int STACK, bool ANY>
__device__ __forceinline__ void traverse_wide(const DevScene &S, const WideScene &WS, const RayP &r, float tmax,
                                              HitRec &h) {
  h.t = tmax;
  h.u = h.v = 0.0f;
  h.prim = INT32_MIN;
  h.inst = -1;
  if (!(tmax > kRayEps)) {
    h.prim = -1;
    return;
  }
  float tn0;
  float bound0 = ANY ? tmax : tmax * kPruneScale;
  if (!slab(r, S.rmin[0], S.rmin[1], S.rmin[2], S.rmax[0], S.rmax[1], S.rmax[2], bound0, tn0)) {
    h.prim = -1;
    return;
  }
  int32_t ref = WS.root;
  int2 stk[STACK];  // (ref, bits of its entry distance): one 8-byte local store per push
  int sp = 0;
  bool done = (ref == kEmptyRef);
  constexpr int F4 = (W == 4) ? 8 : 16;
  // With no axis parallel to the ray (r.par == 0), each axis's near plane is the box minimum
  // when the ray runs up that axis (1/d > 0) and the maximum otherwise, for every box: the slab
  // test's min((mn - o) / d, (mx - o) / d) is that plane's distance, since subtraction and
  // multiplication round monotonically. Loading the near- and far-plane rows of a node by these
  // row offsets leaves one 3-way max and one 3-way min per child instead of three pairwise
  // min/max first; the distances, and so the hits, are the slab test's exactly.
  constexpr int Q = W / 4;
  const int nX = r.ix > 0.0f ? 0 : 3, nY = r.iy > 0.0f ? 1 : 4, nZ = r.iz > 0.0f ? 2 : 5;
  const int fX = 3 - nX, fY = 5 - nY, fZ = 7 - nZ;
  while (!done) {
    if (ref >= 0) {
      const float4 *n = WS.wn + (long long)F4 * ref;
      float bound = ANY ? tmax : h.t * kPruneScale;
      float t[W];
      int32_t c[W];
      if (r.par == 0) {
#pragma unroll
        for (int q = 0; q < Q; ++q) {
          const float4 px = ldg4(n + nX * Q + q), py = ldg4(n + nY * Q + q), pz = ldg4(n + nZ * Q + q);
          const float4 gx = ldg4(n + fX * Q + q), gy = ldg4(n + fY * Q + q), gz = ldg4(n + fZ * Q + q);
          const float4 rf = ldg4(n + 6 * Q + q);
          const float ax[4] = {px.x, px.y, px.z, px.w}, ay[4] = {py.x, py.y, py.z, py.w};
          const float az[4] = {pz.x, pz.y, pz.z, pz.w}, bx[4] = {gx.x, gx.y, gx.z, gx.w};
          const float by[4] = {gy.x, gy.y, gy.z, gy.w}, bz[4] = {gz.x, gz.y, gz.z, gz.w};
          const int32_t rr[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z),
                                 __float_as_int(rf.w)};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const float tnx = (ax[k] - r.ox) * r.ix, tny = (ay[k] - r.oy) * r.iy, tnz = (az[k] - r.oz) * r.iz;
            const float tfx = (bx[k] - r.ox) * r.ix, tfy = (by[k] - r.oy) * r.iy, tfz = (bz[k] - r.oz) * r.iz;
            const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, kRayEps));
            const float tf = fminf(fminf(tfx, tfy), fminf(tfz, bound));
            const bool hk = rr[k] != kEmptyRef && !(tf < tn);
            t[q * 4 + k] = hk ? tn : INFINITY;
            c[q * 4 + k] = hk ? rr[k] : kEmptyRef;
          }
        }
      } else
#pragma unroll
      for (int q = 0; q < W / 4; ++q) {
        float4 mnx = ldg4(n + 0 * (W / 4) + q), mny = ldg4(n + 1 * (W / 4) + q), mnz = ldg4(n + 2 * (W / 4) + q);
        float4 mxx = ldg4(n + 3 * (W / 4) + q), mxy = ldg4(n + 4 * (W / 4) + q), mxz = ldg4(n + 5 * (W / 4) + q);
        float4 rf = ldg4(n + 6 * (W / 4) + q);
        const float ax[4] = {mnx.x, mnx.y, mnx.z, mnx.w}, ay[4] = {mny.x, mny.y, mny.z, mny.w};
        const float az[4] = {mnz.x, mnz.y, mnz.z, mnz.w}, bx[4] = {mxx.x, mxx.y, mxx.z, mxx.w};
        const float by[4] = {mxy.x, mxy.y, mxy.z, mxy.w}, bz[4] = {mxz.x, mxz.y, mxz.z, mxz.w};
        const int32_t rr[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z), __float_as_int(rf.w)};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          float tk;
          bool hk = rr[k] != kEmptyRef && slab(r, ax[k], ay[k], az[k], bx[k], by[k], bz[k], bound, tk);
          t[q * 4 + k] = hk ? tk : INFINITY;
          c[q * 4 + k] = hk ? rr[k] : kEmptyRef;
        }
      }
      sort_children<W>(t, c);
      if (c[0] == kEmptyRef) {
        ref = kEmptyRef;  // nothing hit: pop below
      } else {
#pragma unroll
        for (int k = W - 1; k >= 1; --k) {
          if (c[k] != kEmptyRef) {
            if (sp < STACK) {
              stk[sp] = make_int2(c[k], __float_as_int(t[k]));
              ++sp;
            } else {
              atomicOr(S.status, kStatusStackOverflow);
            }
          }
        }
        ref = c[0];
        continue;
      }
    } else if (ref != kEmptyRef) {
      Work w{0, 0, 0};
      if (leaf_walk<ANY, false>(S, r, ~(int64_t)ref, h, w)) break;
    }
    // pop, dropping entries that now start beyond the best hit
    ref = kEmptyRef;
    while (sp > 0) {
      --sp;
      const int2 e = stk[sp];
      if (!ANY && __int_as_float(e.y) > h.t * kPruneScale) continue;
      ref = e.x;
      break;
    }
    if (ref == kEmptyRef) break;
  }
  if (h.prim == INT32_MIN) {
    h.prim = -1;
    h.inst = -1;
  }
}

}  // namespace nomad_dev
