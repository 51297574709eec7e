// Hybrid packet traversal: persistent warps take 32 consecutive rays; when they are coherent (one
// origin, directions inside a narrow cone: the primary rays of a pinhole view) the warp walks the
// tree as one packet, otherwise each lane runs the per-ray walk of rt_wide.cuh / rt_device.cuh.
//
// Packet walk (warp-uniform control flow): every lane tests the children of the same node against
// its own ray and its own current best hit (the contract's box test and pruning bound); a child is
// visited when any lane hits it (ballot), in the near-first order of the first active lane; leaves
// are tested by every lane. Node and triangle loads are the same address across the warp
// (broadcast). Each lane therefore tests a superset of the boxes and primitives its own walk would
// test, and the closest-hit contract (lowest (t, primitive), pruning margin) makes the result
// independent of visit order and of extra tests: hits are bit-identical to every other variant.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "rt_context.h"

using namespace nomad_dev;

namespace {

constexpr int kPkBlock = 128;
constexpr int kPkWarps = kPkBlock / 32;
constexpr int kPkStack = 128;  // warp stack entries (union walk: at most (W-1) per level)

struct PkArgs {
  const float4 *nodes;  // pair nodes (W = 2) or wide nodes
  int32_t root;
  float cosMin;         // coherence: every direction within this cosine of the leader's
  float originEps;      // coherence: every origin within this distance of the leader's
};

template <int W> struct PkLay;
template <> struct PkLay<2> { static constexpr int F4 = 4; };
template <> struct PkLay<4> { static constexpr int F4 = 8; };
template <> struct PkLay<8> { static constexpr int F4 = 16; };

__device__ __forceinline__ void write_result(bool any, uint64_t i, const HitRec &h, int32_t *hits5, uint8_t *occ) {
  if (any) {
    occ[i] = h.prim >= 0 ? 1 : 0;
  } else {
    int32_t *o = hits5 + 5 * i;
    o[0] = h.inst;
    o[1] = h.prim;
    o[2] = __float_as_int(h.prim >= 0 ? h.t : INFINITY);
    o[3] = __float_as_int(h.u);
    o[4] = __float_as_int(h.v);
  }
}

// The packet walk for the lanes in `lanes` (a warp-uniform mask); `live` is this lane's bit.
template <int W, bool ANY>
__device__ void packet_walk(const DevScene &S, const PkArgs &A, const RayP &r, float tmax, HitRec &h, bool live,
                            unsigned lanes, int32_t *stk) {
  constexpr int F4 = PkLay<W>::F4;
  const unsigned lane = threadIdx.x & 31u;
  bool act = live;  // any-hit lanes leave the packet once occluded
  int sp = 0;
  int32_t ref = A.root;
  for (;;) {
    if (ref >= 0) {
      const float4 *n = A.nodes + (size_t)F4 * ref;
      const float bound = ANY ? tmax : h.t * kPruneScale;
      float t[W];
      int32_t c[W];
      unsigned m[W];
      if constexpr (W == 2) {
        const float4 a = __ldg(n), b = __ldg(n + 1), cc = __ldg(n + 2), d = __ldg(n + 3);
        c[0] = __float_as_int(a.w);
        c[1] = __float_as_int(b.w);
        float t0, t1;
        const bool h0 = act && c[0] != kEmptyRef && slab(r, a.x, a.y, a.z, b.x, b.y, b.z, bound, t0);
        const bool h1 = act && c[1] != kEmptyRef && slab(r, cc.x, cc.y, cc.z, d.x, d.y, d.z, bound, t1);
        t[0] = h0 ? t0 : INFINITY;
        t[1] = h1 ? t1 : INFINITY;
        m[0] = __ballot_sync(lanes, h0);
        m[1] = __ballot_sync(lanes, h1);
      } else {
#pragma unroll
        for (int q = 0; q < W / 4; ++q) {
          const float4 mnx = __ldg(n + 0 * (W / 4) + q), mny = __ldg(n + 1 * (W / 4) + q);
          const float4 mnz = __ldg(n + 2 * (W / 4) + q), mxx = __ldg(n + 3 * (W / 4) + q);
          const float4 mxy = __ldg(n + 4 * (W / 4) + q), mxz = __ldg(n + 5 * (W / 4) + q);
          const float4 rf = __ldg(n + 6 * (W / 4) + q);
          const float ax[4] = {mnx.x, mnx.y, mnx.z, mnx.w}, ay[4] = {mny.x, mny.y, mny.z, mny.w};
          const float az[4] = {mnz.x, mnz.y, mnz.z, mnz.w}, bx[4] = {mxx.x, mxx.y, mxx.z, mxx.w};
          const float by[4] = {mxy.x, mxy.y, mxy.z, mxy.w}, bz[4] = {mxz.x, mxz.y, mxz.z, mxz.w};
          const int32_t rr[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z),
                                 __float_as_int(rf.w)};
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            float tk;
            const bool hk = act && rr[k] != kEmptyRef && slab(r, ax[k], ay[k], az[k], bx[k], by[k], bz[k], bound, tk);
            t[q * 4 + k] = hk ? tk : INFINITY;
            c[q * 4 + k] = rr[k];
            m[q * 4 + k] = __ballot_sync(lanes, hk);
          }
        }
      }
      // near-first order of the first lane that hit anything (warp-uniform)
      unsigned anyHit = 0;
#pragma unroll
      for (int k = 0; k < W; ++k) anyHit |= m[k];
      if (anyHit == 0) {
        ref = sp > 0 ? stk[--sp] : kEmptyRef;
        if (ref == kEmptyRef) break;
        continue;
      }
      const int leader = __ffs(anyHit) - 1;
      float lt[W];
      int32_t ord[W];
#pragma unroll
      for (int k = 0; k < W; ++k) {
        lt[k] = __shfl_sync(lanes, t[k], leader);
        // children no lane hit sort last and are skipped below
        if (m[k] == 0) lt[k] = INFINITY;
        ord[k] = k;
      }
      sort_children<W>(lt, ord);
      int32_t next = kEmptyRef;
#pragma unroll
      for (int k = W - 1; k >= 0; --k) {
        const int j = ord[k];
        if (m[j] == 0) continue;
        if (next != kEmptyRef && sp < kPkStack) {
          if (lane == 0) stk[sp] = next;
          ++sp;
        } else if (next != kEmptyRef) {
          if (lane == 0) atomicOr(S.status, kStatusStackOverflow);
        }
        next = c[j];
      }
      __syncwarp(lanes);
      ref = next;
      continue;
    }
    // leaf: every live lane tests its records
    {
      int64_t k = ~(int64_t)ref;
      for (;;) {
        const float4 *q = S.tri + 3 * k;
        const float4 Av = __ldg(q), Bv = __ldg(q + 1), Cv = __ldg(q + 2);
        const int32_t pid = __float_as_int(Av.w);
        const int32_t meta = __float_as_int(Cv.w);
        if (act && pid >= 0 && test_prim(S, r, Av, Bv, Cv, pid, meta & 0xff, h) && ANY) act = false;
        if (meta & kLastInLeaf) break;
        ++k;
      }
    }
    if (ANY && __ballot_sync(lanes, act) == 0) break;
    __syncwarp(lanes);
    if (sp == 0) break;
    ref = stk[--sp];
  }
  __syncwarp(lanes);
}

template <int W, bool ANY>
__global__ void __launch_bounds__(kPkBlock) k_trace_packet(DevScene S, WideScene WS, PkArgs A,
                                                           const float4 *__restrict__ rays, uint64_t n,
                                                           const uint32_t *__restrict__ lenDev,
                                                           unsigned long long *__restrict__ cursor,
                                                           int32_t *__restrict__ hits5, uint8_t *__restrict__ occ,
                                                           uint32_t *__restrict__ counts) {
  __shared__ int32_t sstk[kPkWarps][kPkStack];
  int32_t *stk = sstk[threadIdx.x >> 5];
  const uint64_t N = lenDev ? (uint64_t)*lenDev : n;
  const unsigned lane = threadIdx.x & 31u;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(cursor, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= N) break;
    const uint64_t i = base + lane;
    const bool has = i < N;
    float4 ra = make_float4(0.f, 0.f, 0.f, 0.f), rb = make_float4(0.f, 0.f, 0.f, 0.f);
    if (has) {
      ra = __ldg(rays + 2 * i);
      rb = __ldg(rays + 2 * i + 1);
    }
    const RayP r = prep_ray(ra, rb);
    const float tmax = rb.w;
    // a lane joins the walk when its ray can hit the root box
    float tn0;
    const bool live = has && tmax > kRayEps && A.root != kEmptyRef &&
                      slab(r, S.rmin[0], S.rmin[1], S.rmin[2], S.rmax[0], S.rmax[1], S.rmax[2],
                           ANY ? tmax : tmax * kPruneScale, tn0);
    // coherence against the first lane: same origin (within originEps), direction within the cone
    const float lox = __shfl_sync(0xffffffffu, ra.x, 0), loy = __shfl_sync(0xffffffffu, ra.y, 0);
    const float loz = __shfl_sync(0xffffffffu, ra.z, 0);
    const float ldx = __shfl_sync(0xffffffffu, rb.x, 0), ldy = __shfl_sync(0xffffffffu, rb.y, 0);
    const float ldz = __shfl_sync(0xffffffffu, rb.z, 0);
    const float ddot = ldx * rb.x + ldy * rb.y + ldz * rb.z;
    const float dl = sqrtf((ldx * ldx + ldy * ldy + ldz * ldz) * (rb.x * rb.x + rb.y * rb.y + rb.z * rb.z));
    const bool coh = !has || (fabsf(ra.x - lox) <= A.originEps && fabsf(ra.y - loy) <= A.originEps &&
                              fabsf(ra.z - loz) <= A.originEps && ddot >= A.cosMin * dl);
    HitRec h;
    h.t = tmax;
    h.u = h.v = 0.0f;
    h.prim = INT32_MIN;
    h.inst = -1;
    if (__all_sync(0xffffffffu, coh)) {
      const unsigned lanes = 0xffffffffu;
      if (__any_sync(lanes, live)) packet_walk<W, ANY>(S, A, r, tmax, h, live, lanes, stk);
      if (h.prim == INT32_MIN) {
        h.prim = -1;
        h.inst = -1;
      }
    } else if (has) {
      if (W == 2) {
        Work w{0, 0, 0};
        traverse<64, ANY, false>(S, r, tmax, h, w);
      } else {
        traverse_wide<W, (W == 8 ? 96 : 64), ANY>(S, WS, r, tmax, h);
      }
    }
    if (has) write_result(ANY, i, h, hits5, occ);
    if (!ANY && counts) {
      const int32_t key = (has && h.prim >= 0) ? h.inst : -1;
      const unsigned peers = __match_any_sync(0xffffffffu, key);
      if (key >= 0 && (int)lane == __ffs(peers) - 1) atomicAdd(counts + key, (uint32_t)__popc(peers));
    }
    __syncwarp();
  }
}

template <int W, bool ANY>
nomad_status launch_pk(nomad_ctx *ctx, const WideScene &WS, const PkArgs &A, const float4 *rays, uint64_t n,
                       const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5, uint8_t *occ,
                       uint32_t *counts, cudaStream_t s) {
  auto kern = k_trace_packet<W, ANY>;
  int perSm = 0;
  NOMAD_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kPkBlock, 0));
  uint64_t blocks = (uint64_t)ctx->smCount * (uint64_t)std::max(perSm, 1);
  blocks = std::max<uint64_t>(1, std::min(blocks, (n + kPkBlock - 1) / kPkBlock));
  NOMAD_CUDA(ctx, cudaMemsetAsync(cursor, 0, 8, s));
  kern<<<(unsigned)blocks, kPkBlock, 0, s>>>(ctx->scene, WS, A, rays, n, lenDev, cursor, hits5, occ, counts);
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

}  // namespace

nomad_status nomad_trace_packet(nomad_ctx *ctx, const nomad_traversal &cfg, bool any, const float4 *rays, uint64_t n,
                                const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5, uint8_t *occ,
                                uint32_t *counts, cudaStream_t s) {
  PkArgs A;
  const float *mn = ctx->layout.rootMin, *mx = ctx->layout.rootMax;
  const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  A.originEps = 1e-6f * std::sqrt(dx * dx + dy * dy + dz * dz);
  A.cosMin = 0.9995f;  // about 1.8 degrees
  WideScene WS{nullptr, kEmptyRef};
  if (cfg.width == 2) {
    A.nodes = ctx->scene.pn;
    A.root = ctx->scene.rootRef;
  } else {
    WS = ctx->ws[cfg.width == 4 ? 0 : 1];
    A.nodes = WS.wn;
    A.root = WS.root;
  }
  switch (cfg.width) {
    case 2: return any ? launch_pk<2, true>(ctx, WS, A, rays, n, lenDev, cursor, hits5, occ, counts, s)
                       : launch_pk<2, false>(ctx, WS, A, rays, n, lenDev, cursor, hits5, occ, counts, s);
    case 4: return any ? launch_pk<4, true>(ctx, WS, A, rays, n, lenDev, cursor, hits5, occ, counts, s)
                       : launch_pk<4, false>(ctx, WS, A, rays, n, lenDev, cursor, hits5, occ, counts, s);
    case 8: return any ? launch_pk<8, true>(ctx, WS, A, rays, n, lenDev, cursor, hits5, occ, counts, s)
                       : launch_pk<8, false>(ctx, WS, A, rays, n, lenDev, cursor, hits5, occ, counts, s);
    default: return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "width must be 2, 4 or 8");
  }
}
