// Residency on the device: per-object hit history and features, policy scores, byte-budgeted
// selection, TLAS patching and the light CDF that follows the resident set.
//
// Restated from the reference:
//   * light CDF over active emissive primitives, weight = area * power * luminance(colour)
//     (Renderer.cpp:5161-5211, primitiveArea :1462-1480);
//   * decayed ray-hit score, score = score * rayHitDecay + hits (processRayHitCounters,
//     Renderer.cpp:8449-8451), adjusted as updateRayHitBudget does (RendererResidency.cpp:
//     2833-2840: off-screen objects without hits drop to 0, off-screen objects with hits keep
//     lerp(0.5, 0.2, memoryPressure), visible objects with no score get 1);
//   * selection in score order with ties to the lower index (:2883-2896), a visibility reserve
//     of ceil(N * (0.02 + 0.06 * motion)) visible objects (:2908-2923), min_active always kept
//     (:2925-2926) and a per-step toggle budget applied in index order (:2930-2946).
// Changes for the B200 build: the unit is the object (the reference toggles primitives), and the
// target is a geometry byte budget rather than a primitive fraction (greedy in score order,
// skipping objects that do not fit).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <vector>

#include "pt_lights.cuh"
#include "residency_features.cuh"
#include "rt_context.h"

using namespace nomad_dev;

namespace {

using nomad_res::CamDev;
using nomad_res::FeatArgs;
using nomad_res::kHist;
constexpr uint32_t kMaxSelectObjects = 16384;

__global__ void k_features(FeatArgs A, float *__restrict__ keys) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= A.n) return;
  float f[NOMAD_FEATURES];
  keys[o] = nomad_res::object_features(A, o, f);
}

// The per-object Beta hit-probability posterior of processRayHitCounters (Renderer.cpp:
// 8420-8522, restated in the same float operation order), one thread per object, after the
// feature pass of the same step (which stored the step's closest hits in the history and the
// visibility flag). post holds kPostWords words per object: alpha, beta, probability (clamped),
// variance, posterior mass, exploration score (f32), idle steps, hits, rays tested (u32).
struct PostArgs {
  uint32_t n, frame;
  const uint32_t *hist;
  uint32_t *tests;
  const uint8_t *visible, *res;
  float *post;
  float decay, hitDecay, maxMass, idleDecay, threshold;
  int clampMass;
  uint32_t idleFrames;
  float *keys;       // ray-hit keys to multiply by the prior weight, or null
  float priorScale;
};

__device__ __forceinline__ float renormalize_posterior(float &alpha, float &beta, const PostArgs &A) {
  constexpr float kMinMass = 1.0e-3f;
  float sum = alpha + beta;
  if (!(sum > 0.0f)) {
    alpha = beta = kMinMass * 0.5f;
    sum = kMinMass;
  } else if (sum < kMinMass) {
    const float scale = kMinMass / sum;
    alpha *= scale;
    beta *= scale;
    sum = kMinMass;
  }
  if (A.clampMass && sum > A.maxMass) {
    const float scale = A.maxMass / sum;
    alpha *= scale;
    beta *= scale;
    sum = A.maxMass;
  }
  return sum;
}

__device__ __forceinline__ float clamp01(float v) { return v < 0.0f ? 0.0f : (1.0f < v ? 1.0f : v); }
__device__ __forceinline__ float maxf_ref(float a, float b) { return a < b ? b : a; }  // std::max

__global__ void k_posterior(PostArgs A) {
  const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= A.n) return;
  float *p = A.post + (size_t)o * kPostWords;
  uint32_t *pu = reinterpret_cast<uint32_t *>(p);
  const uint32_t h = A.hist[o * kHist + A.frame % kHist];
  const uint32_t t = A.tests[o];
  A.tests[o] = 0;
  const float success = (float)h, rays = (float)t;
  const bool visible = A.visible[o] != 0, active = A.res[o] != 0;
  const float failure = maxf_ref(rays - success, 0.0f);
  float alpha = p[0] * A.decay + success;
  float beta = p[1] * A.decay + failure;
  float sum = alpha + beta;
  float prob = sum > 0.0f ? alpha / sum : 0.5f;
  uint32_t idle = pu[6];
  if (t == 0) {
    const bool grace = A.idleFrames > 0 && (visible || active) && idle < A.idleFrames;
    float cooling = A.decay;
    bool apply = true;
    if (grace) {
      if (A.idleDecay >= 0.999f) apply = false;
      else cooling = A.idleDecay;
    }
    if (apply) {
      const float cp = clamp01(prob * cooling);
      float cm = maxf_ref(sum, 1.0e-3f);
      if (A.clampMass && cm > A.maxMass) cm = A.maxMass;
      alpha = cp * cm;
      beta = maxf_ref(cm - alpha, 0.0f);
    }
  }
  sum = renormalize_posterior(alpha, beta, A);
  prob = sum > 0.0f ? alpha / sum : 0.5f;
  const float clamped = clamp01(prob);
  float var = 0.0f;
  if (sum > 1.0f) var = (alpha * beta) / ((sum * sum) * (sum + 1.0f));
  float ex = p[5] * A.decay;
  if (t > 0) {
    idle = 0;
    if (clamped < A.threshold) ex += rays;
    else ex *= A.hitDecay;
  } else {
    if (idle < 0xffffffffu) ++idle;
    ex *= A.hitDecay;
    if (visible || active) ex = maxf_ref(ex, 1.0f);  // kIdleVisibleExploreSeed
  }
  p[0] = alpha;
  p[1] = beta;
  p[2] = clamped;
  p[3] = maxf_ref(var, 0.0f);
  p[4] = sum;
  p[5] = ex;
  pu[6] = idle;
  pu[7] = h;
  pu[8] = t;
  // ray-hit prior (RendererResidency.cpp:2842-2861, rayHitPriorFavorHighProbability off)
  if (A.keys && A.priorScale > 0.0f) {
    float w = 1.0f + (clamped - 0.5f) * A.priorScale * 1.0f;
    w = w < 0.25f ? 0.25f : (1.0f < w ? 1.0f : w);
    A.keys[o] *= w;
  }
}

__device__ __forceinline__ unsigned long long sort_key(float s, uint32_t idx) {
  if (!(s == s) || isinf(s)) s = 0.0f;  // sanitize like sanitizeSortValue
  uint32_t b = __float_as_uint(s);
  b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);  // ascending float -> ascending uint
  return ((unsigned long long)(~b) << 32) | idx;     // descending score, then ascending index
}

// Block-wide exclusive scan of one u32 per thread (1024 threads); returns this thread's prefix
// and writes the total to *total (shared).
__device__ __forceinline__ uint32_t block_exscan(uint32_t v, uint32_t *warpSums, uint32_t *total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if ((int)lane >= d) x += y;
  }
  if (lane == 31) warpSums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = warpSums[lane];
    uint32_t z = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, z, d);
      if ((int)lane >= d) z += y;
    }
    warpSums[lane] = z - w;  // exclusive prefix of the warp totals
    if (lane == 31) *total = z;
  }
  __syncthreads();
  const uint32_t r = warpSums[warp] + x - v;
  __syncthreads();
  return r;
}

// Block-wide exclusive scan of one u64 per thread (1024 threads); writes the total to *total.
__device__ __forceinline__ unsigned long long block_exscan64(unsigned long long v, unsigned long long *warpSums,
                                                             unsigned long long *total) {
  const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  unsigned long long x = v;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const unsigned long long y = __shfl_up_sync(0xffffffffu, x, d);
    if ((int)lane >= d) x += y;
  }
  if (lane == 31) warpSums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const unsigned long long w = warpSums[lane];
    unsigned long long z = w;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, z, d);
      if ((int)lane >= d) z += y;
    }
    warpSums[lane] = z - w;
    if (lane == 31) *total = z;
  }
  __syncthreads();
  const unsigned long long r = warpSums[warp] + x - v;
  __syncthreads();
  return r;
}

// After the sort each key holds (object bytes / 4) in its high word and the object in its low
// word. Object bytes are 32 per node + 196 per primitive, so always a multiple of 4, and
// "used + b <= budget" holds exactly when "used/4 + b/4 <= budget/4" (rounded down).
__device__ __forceinline__ uint32_t key_obj(unsigned long long k) { return (uint32_t)(k & 0xffffffffu); }
__device__ __forceinline__ unsigned long long key_b4(unsigned long long k) { return k >> 32; }

// Greedy fill in sorted order from position `from` by one warp: candidates are taken while they
// fit, skipping those that do not (the sequential rule), 32 positions at a time. Each round
// first drops lanes that cannot fit on their own, then accepts the longest run of candidates
// whose running total fits; the first candidate past that run is skipped.
__device__ void warp_greedy(uint32_t from, uint32_t n, const unsigned long long *sk, unsigned long long budget4,
                            bool unlimited, const uint8_t *cand, uint8_t *dsel, unsigned long long *used4) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long u = *used4;
  for (uint32_t base = from; base < n; base += 32) {
    const uint32_t k = base + lane;
    bool c = k < n && cand[k];
    const unsigned long long b = c ? key_b4(sk[k]) : 0ull;
    for (;;) {
      const unsigned long long rem = unlimited ? ~0ull : (u > budget4 ? 0ull : budget4 - u);
      if (c && b > rem) c = false;
      if (__ballot_sync(0xffffffffu, c) == 0) break;
      unsigned long long p = c ? b : 0ull;  // inclusive prefix of candidate bytes
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, p, d);
        if ((int)lane >= d) p += y;
      }
      const unsigned fail = __ballot_sync(0xffffffffu, c && p > rem);
      const int f = fail ? __ffs(fail) - 1 : 32;
      if (c && (int)lane < f) dsel[k] = 1;
      const unsigned long long pf = __shfl_sync(0xffffffffu, p, f < 32 ? f : 31);
      const unsigned long long bf = __shfl_sync(0xffffffffu, b, f < 32 ? f : 31);
      u += f < 32 ? pf - bf : pf;
      c = c && (int)lane > f;
    }
  }
  if (lane == 0) *used4 = u;
}

struct SelectShared {
  unsigned long long warpSums64[32];
  unsigned long long total64;
  unsigned long long used4;
  unsigned long long add4;
  uint32_t warpSums[32];
  uint32_t total;
  uint32_t first;
};

// One budget walk over the candidates (cand[k] = 1) in sorted order, with the whole block: a
// block scan of candidate bytes finds the first candidate that no longer fits; every candidate
// before it is taken at once, that one is skipped, and one warp finishes the walk after it
// (where the remaining budget is below that candidate's size, so most objects drop at once).
__device__ void budget_walk(uint32_t n, uint32_t npow2, const unsigned long long *sk, unsigned long long budget4,
                            bool unlimited, const uint8_t *cand, uint8_t *dsel, SelectShared &sh) {
  const uint32_t per = (npow2 + blockDim.x - 1) / blockDim.x;
  const uint32_t k0 = threadIdx.x * per, k1 = min(k0 + per, n);
  unsigned long long seg = 0;
  for (uint32_t k = k0; k < k1; ++k)
    if (cand[k]) seg += key_b4(sk[k]);
  if (threadIdx.x == 0) sh.first = npow2;
  const unsigned long long excl = block_exscan64(seg, sh.warpSums64, &sh.total64);  // syncs inside
  const unsigned long long u0 = sh.used4;
  const unsigned long long rem = unlimited ? ~0ull : (u0 > budget4 ? 0ull : budget4 - u0);
  unsigned long long run = excl;
  for (uint32_t k = k0; k < k1; ++k) {
    if (!cand[k]) continue;
    run += key_b4(sk[k]);
    if (run > rem) {
      atomicMin(&sh.first, k);
      break;
    }
  }
  __syncthreads();
  const uint32_t R = sh.first;
  unsigned long long before = excl;  // candidate bytes before R inside this segment
  for (uint32_t k = k0; k < k1 && k < R; ++k)
    if (cand[k]) {
      dsel[k] = 1;
      before += key_b4(sk[k]);
    }
  if (R < npow2 && k0 <= R && R < k0 + per) sh.add4 = before;  // the segment holding R
  if (R >= npow2 && threadIdx.x == 0) sh.add4 = sh.total64;
  __syncthreads();
  if (threadIdx.x == 0) sh.used4 = u0 + sh.add4;
  __syncthreads();
  if (R + 1 < n && threadIdx.x < 32) warp_greedy(R + 1, n, sk, budget4, unlimited, cand, dsel, &sh.used4);
  __syncthreads();
}

// Light CDF over the emissive primitives whose primitive is active and whose object is
// resident, summed sequentially in primitive order (one thread; the flags are gathered by the
// block first). Also writes the per-primitive light pdf used by ReSTIR. Called by one block.
__device__ void lights_rebuild(const uint4 *__restrict__ em, uint32_t ne, const uint8_t *__restrict__ primAct,
                               const uint8_t *objRes, uint32_t *__restrict__ idx, float *__restrict__ cdf,
                               float *__restrict__ pdf, LightMeta *__restrict__ meta, uint8_t *on, float &total_s,
                               uint32_t &count_s, const float4 *__restrict__ prims, const float4 *__restrict__ mats,
                               float4 *__restrict__ rec) {
  if (threadIdx.x == 0) {
    total_s = 0.0f;
    count_s = 0;
  }
  __syncthreads();
  for (uint32_t base = 0; base < ne; base += 4096) {
    uint32_t m = min(4096u, ne - base);
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) {
      uint4 e = em[base + i];
      on[i] = primAct[e.x] && objRes[e.z];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      float total = total_s;
      uint32_t c = count_s;
      for (uint32_t i = 0; i < m; ++i) {
        uint4 e = em[base + i];
        pdf[e.x] = 0.0f;
        if (!on[i]) continue;
        total += __uint_as_float(e.y);
        idx[c] = e.x;
        cdf[c] = total;
        ++c;
      }
      total_s = total;
      count_s = c;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    float total = total_s;
    uint32_t c = count_s;
    meta->count = c;
    meta->total = total;
    float prev = 0.0f;
    for (uint32_t k = 0; k < c; ++k) {
      float w = cdf[k] - prev;
      prev = cdf[k];
      if (w > 0.0f && total > 0.0f) pdf[idx[k]] = w / total;
    }
  }
  __syncthreads();
  // light records of the new CDF (the weight of slot k is cdf[k] - cdf[k-1], as samplers read it)
  const uint32_t c = count_s;
  const float total = total_s;
  for (uint32_t k = threadIdx.x; k < c; k += blockDim.x) {
    const float prev = k > 0 ? cdf[k - 1] : 0.0f;
    nomad_pt::light_record(prims, mats, idx[k], cdf[k] - prev, total, rec + 5ull * k);
  }
}

__global__ void __launch_bounds__(1024) k_lights_rebuild(const uint4 *__restrict__ em, uint32_t ne,
                                                         const uint8_t *__restrict__ primAct,
                                                         const uint8_t *__restrict__ objRes,
                                                         uint32_t *__restrict__ idx, float *__restrict__ cdf,
                                                         float *__restrict__ pdf, LightMeta *__restrict__ meta,
                                                         const float4 *__restrict__ prims,
                                                         const float4 *__restrict__ mats, float4 *__restrict__ rec) {
  __shared__ uint8_t on[4096];
  __shared__ float total_s;
  __shared__ uint32_t count_s;
  lights_rebuild(em, ne, primAct, objRes, idx, cdf, pdf, meta, on, total_s, count_s, prims, mats, rec);
}

// Wide-layout instance slots that one step rewrites (4- and 8-wide).
struct WidePatch {
  int32_t *arena;
  size_t base[2];
  uint32_t fpn[2], width[2];
  const long long *slot[2];
  const int32_t *ref[2];
};

struct LightArgs {
  const uint4 *em;
  uint32_t ne;
  const uint8_t *primAct;
  uint32_t *idx;
  float *cdf, *pdf;
  LightMeta *meta;
  const float4 *prims, *mats;
  float4 *rec;
};

// Single block of 1024 threads, the whole residency decision of one step: sort by score, select
// under the budget (min_active, visibility reserve, fill), apply toggles in index order, patch the
// instance links of the pair and wide layouts, and rebuild the light CDF over the new resident set.
__global__ void __launch_bounds__(1024) k_select(uint32_t n, uint32_t npow2, uint32_t policy,
                                                 const float *__restrict__ keys, const uint8_t *__restrict__ visible,
                                                 const unsigned long long *__restrict__ bytes,
                                                 unsigned long long budget, uint32_t reserve, uint32_t minActive,
                                                 uint32_t maxToggles, float resBonus, uint8_t *__restrict__ desired,
                                                 uint8_t *__restrict__ res, const long long *__restrict__ slot,
                                                 const int32_t *__restrict__ blasRef, int32_t *__restrict__ pnodeWords,
                                                 uint32_t *__restrict__ misc, WidePatch wp, LightArgs la) {
  extern __shared__ unsigned long long sk[];
  uint8_t *dsel = reinterpret_cast<uint8_t *>(sk + npow2);  // selected, by sorted position
  uint8_t *cand = dsel + npow2;                             // candidates of the current walk
  __shared__ SelectShared sh;
  __shared__ uint8_t on[4096];
  __shared__ float ltotal;
  __shared__ uint32_t lcount;
  for (uint32_t i = threadIdx.x; i < npow2; i += blockDim.x) {
    float k = 1.0f;
    if (i < n && policy != NOMAD_POLICY_ALWAYS) {
      k = keys[i];
      if (resBonus != 0.0f && res[i]) k = k + resBonus * fabsf(k);  // hysteresis for resident objects
    }
    sk[i] = i < n ? sort_key(k, i) : ~0ull;
  }
  if (threadIdx.x == 0) {
    sh.used4 = 0;
    misc[1] = 0;
  }
  __syncthreads();
  for (uint32_t k = 2; k <= npow2; k <<= 1) {
    for (uint32_t j = k >> 1; j > 0; j >>= 1) {
      for (uint32_t i = threadIdx.x; i < npow2; i += blockDim.x) {
        uint32_t l = i ^ j;
        if (l > i) {
          unsigned long long a = sk[i], b = sk[l];
          bool up = (i & k) == 0;
          if ((a > b) == up) {
            sk[i] = b;
            sk[l] = a;
          }
        }
      }
      __syncthreads();
    }
  }
  // sorted keys -> (bytes / 4, object)
  for (uint32_t k = threadIdx.x; k < npow2; k += blockDim.x) {
    const uint32_t o = (uint32_t)(sk[k] & 0xffffffffu);
    sk[k] = k < n ? ((unsigned long long)(bytes[o] >> 2) << 32) | o : 0ull;
  }
  __syncthreads();
  const bool unlimited = budget == 0 || policy == NOMAD_POLICY_ALWAYS;
  const unsigned long long budget4 = budget >> 2;
  // min_active: the best-scored objects stay whatever the budget
  for (uint32_t k = threadIdx.x; k < npow2; k += blockDim.x) {
    const bool m = k < n && k < minActive;
    dsel[k] = m ? 1 : 0;
    if (m) atomicAdd(&sh.used4, key_b4(sk[k]));
  }
  __syncthreads();
  // visibility reserve: the first `reserve` visible objects in score order (a contiguous segment
  // of sorted positions per thread, so the scan keeps the sorted order)
  const uint32_t per = (npow2 + blockDim.x - 1) / blockDim.x;
  const uint32_t k0 = threadIdx.x * per;
  uint32_t nv = 0;
  for (uint32_t k = k0; k < k0 + per && k < n; ++k) nv += visible[key_obj(sk[k])] ? 1u : 0u;
  uint32_t before = block_exscan(nv, sh.warpSums, &sh.total);
  for (uint32_t k = k0; k < k0 + per && k < npow2; ++k) {
    bool c = false;
    if (k < n && visible[key_obj(sk[k])]) {
      c = before < reserve && !dsel[k];
      ++before;
    }
    cand[k] = c ? 1 : 0;
  }
  __syncthreads();
  budget_walk(n, npow2, sk, budget4, unlimited, cand, dsel, sh);
  // fill in score order
  for (uint32_t k = threadIdx.x; k < npow2; k += blockDim.x) cand[k] = (k < n && !dsel[k]) ? 1 : 0;
  __syncthreads();
  budget_walk(n, npow2, sk, budget4, unlimited, cand, dsel, sh);
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) desired[key_obj(sk[k])] = dsel[k];
  __syncthreads();
  // toggles in index order, the first max_toggles of them when bounded
  uint32_t nd = 0;
  for (uint32_t o = k0; o < k0 + per && o < n; ++o) nd += desired[o] != res[o] ? 1u : 0u;
  uint32_t rank = block_exscan(nd, sh.warpSums, &sh.total);
  for (uint32_t o = k0; o < k0 + per && o < n; ++o) {
    const uint8_t want = desired[o];
    if (want == res[o]) continue;
    const bool apply = maxToggles == 0 || rank < maxToggles;
    ++rank;
    if (!apply) continue;
    res[o] = want;
    const long long s = slot[o];
    const int32_t ref = want ? blasRef[o] : kEmptyRef;
    if (s >= 0) {
      pnodeWords[(s / 2) * 16 + ((s & 1) ? 7 : 3)] = ref;
    } else if (s == -1) {
      misc[1] = 1;
      misc[2] = want;
    }
    for (int w = 0; w < 2; ++w) {
      if (!wp.width[w]) continue;
      const long long ws = wp.slot[w][o];
      if (ws < 0) continue;
      wp.arena[wp.base[w] + (size_t)(ws / wp.width[w]) * wp.fpn[w] + 6 * wp.width[w] + (size_t)(ws % wp.width[w])] =
          want ? wp.ref[w][o] : kEmptyRef;
    }
  }
  if (threadIdx.x == 0) {
    misc[0] = maxToggles == 0 ? sh.total : min(sh.total, maxToggles);
    misc[4] = misc[3];
    misc[3] = 0;
  }
  __syncthreads();  // res[] complete for the light rebuild
  lights_rebuild(la.em, la.ne, la.primAct, res, la.idx, la.cdf, la.pdf, la.meta, on, ltotal, lcount, la.prims, la.mats,
                 la.rec);
}

float luminance_host(const float *c) { return c[0] * 0.2126f + c[1] * 0.7152f + c[2] * 0.0722f; }

}  // namespace

// Called at scene upload: per-object device arrays, emissive list, bytes, bounds.
nomad_status nomad_residency_init(nomad_ctx *ctx) {
  auto &R = ctx->res;
  const auto &L = ctx->layout;
  const uint32_t N = ctx->objectCount, P = ctx->primCount;
  // a new scene starts the host-side policies afresh
  R.primHitsOn = false;
  R.primHitsHost.clear();
  R.primCooldown.clear();
  R.primStep = 0;
  R.primScore.clear();
  R.primSphere.clear();
  R.primVisible.clear();
  R.primRebuild = 0;
  R.lodOn = false;
  R.fallbackSteps = 0;
  R.objCooldown.clear();
  R.lodDist.clear();
  R.lodFlags.clear();
  NOMAD_CUDA(ctx, R.objSlot.reserve((size_t)N * 8));
  NOMAD_CUDA(ctx, R.objBlasRef.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.objRes.reserve(N));
  NOMAD_CUDA(ctx, R.primAct.reserve(P));
  NOMAD_CUDA(ctx, R.bounds.reserve((size_t)N * 16));
  NOMAD_CUDA(ctx, R.bytes.reserve((size_t)N * 8));
  NOMAD_CUDA(ctx, R.tris.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.emit.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.score.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.hist.reserve((size_t)N * kHist * 4));
  NOMAD_CUDA(ctx, R.lastHit.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.prevDist.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.visible.reserve(N));
  NOMAD_CUDA(ctx, R.features.reserve((size_t)N * NOMAD_FEATURES * 4));
  NOMAD_CUDA(ctx, R.keys.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, R.desired.reserve(N));
  NOMAD_CUDA(ctx, R.misc.reserve(64));
  NOMAD_CUDA(ctx, cudaMemcpy(R.objSlot.p, L.objSlot.data(), (size_t)N * 8, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(R.objBlasRef.p, L.objBlasRef.data(), (size_t)N * 4, cudaMemcpyHostToDevice));
  for (DeviceBuf *b : {&R.score, &R.hist, &R.lastHit, &R.prevDist, &R.misc})
    NOMAD_CUDA(ctx, cudaMemset(b->p, 0, b->bytes));
  // bytes per object: 32 per BLAS node + 196 per primitive; bounds as centre + radius
  std::vector<uint32_t> nodes(N, 0);
  {
    std::vector<std::pair<int32_t, uint32_t>> roots;
    for (uint32_t o = 0; o < N; ++o)
      if (L.objRootNode[o] >= 0) roots.push_back({L.objRootNode[o], o});
    std::sort(roots.begin(), roots.end());
    // every object's nodes are one block: root first (pre-order) or root last (post-order)
    for (size_t i = 0; i < roots.size(); ++i) {
      if (L.blasPostOrder) {
        const uint32_t begin = i ? (uint32_t)roots[i - 1].first + 1 : 0u;
        nodes[roots[i].second] = (uint32_t)roots[i].first + 1 - begin;
      } else {
        const uint32_t end = i + 1 < roots.size() ? (uint32_t)roots[i + 1].first : R.bvhNodeCount;
        nodes[roots[i].second] = end - (uint32_t)roots[i].first;
      }
    }
  }
  R.hostBytes.assign(N, 0);
  std::vector<float4> bounds(N);
  std::vector<uint32_t> tris(N, 0);
  std::vector<float> emit(N, 0.0f);
  const float *Pp = ctx->hostPrims.data();
  const float *M = ctx->hostMaterials.data();
  std::vector<uint4> em;
  for (uint32_t o = 0; o < N; ++o) {
    const nomad_instance_record &r = ctx->instances[o];
    R.hostBytes[o] = 32ull * nodes[o] + 196ull * r.primitive_count;
    // the selection kernel packs bytes / 4 into 32 bits
    if (R.hostBytes[o] >= (1ull << 34))
      return nomad_fail(ctx, NOMAD_ERR_LIMIT, "an object holds 16 GB or more of geometry");
    tris[o] = r.primitive_count;
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t p = r.primitive_base; p < r.primitive_base + r.primitive_count; ++p) {
      const float *g = Pp + 28ull * p;
      for (int v = 0; v < 3; ++v)
        for (int k = 0; k < 3; ++k) {
          float c = g[v * 4 + k];
          int type = (int)g[3];
          if (type != 1 && v > 0) c = g[k];  // spheres / rectangles: use the centre
          mn[k] = std::min(mn[k], c);
          mx[k] = std::max(mx[k], c);
        }
    }
    float cx = 0.5f * (mn[0] + mx[0]), cy = 0.5f * (mn[1] + mx[1]), cz = 0.5f * (mn[2] + mx[2]);
    float ex = mx[0] - cx, ey = mx[1] - cy, ez = mx[2] - cz;
    bounds[o] = make_float4(cx, cy, cz, std::sqrt(ex * ex + ey * ey + ez * ez));
  }
  // emissive primitives with their static weights (area * strength), in primitive order
  for (uint32_t i = 0; i < P; ++i) {
    const float *m = M + 20ull * i;
    float strength = m[11] * luminance_host(m + 8);
    if (!(strength > 0.0f)) continue;
    const float *g = Pp + 28ull * i;
    int type = (int)g[3];
    float area = 0.0f;
    if (type == 0) {
      float r = g[4];
      area = 4.0f * 3.14159265358979323846f * r * r;
    } else {
      float ax, ay, az, bx, by, bz;
      if (type == 1) {
        ax = g[4] - g[0]; ay = g[5] - g[1]; az = g[6] - g[2];
        bx = g[8] - g[0]; by = g[9] - g[1]; bz = g[10] - g[2];
      } else {
        ax = g[4]; ay = g[5]; az = g[6];
        bx = g[8]; by = g[9]; bz = g[10];
      }
      float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
      float len = std::sqrt(cx * cx + cy * cy + cz * cz);
      area = type == 1 ? 0.5f * len : 4.0f * len;
    }
    if (!(area > 0.0f)) continue;
    float w = area * strength;
    if (!(w > 0.0f)) continue;
    uint32_t wb;
    std::memcpy(&wb, &w, 4);
    uint32_t obj = (uint32_t)ctx->layout.primObject[i];
    em.push_back(make_uint4(i, wb, obj, 0));
    emit[obj] += w;
  }
  R.emissiveCount = (uint32_t)em.size();
  NOMAD_CUDA(ctx, R.emissive.reserve(std::max<size_t>(1, em.size()) * 16));
  if (!em.empty()) NOMAD_CUDA(ctx, cudaMemcpy(R.emissive.p, em.data(), em.size() * 16, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(R.bytes.p, R.hostBytes.data(), (size_t)N * 8, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(R.bounds.p, bounds.data(), (size_t)N * 16, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(R.tris.p, tris.data(), (size_t)N * 4, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(R.emit.p, emit.data(), (size_t)N * 4, cudaMemcpyHostToDevice));
  FrameState &F = ctx->frame;
  NOMAD_CUDA(ctx, F.lightIdx.reserve(std::max<size_t>(1, em.size()) * 4));
  NOMAD_CUDA(ctx, F.lightRec.reserve(std::max<size_t>(1, em.size()) * 80));
  NOMAD_CUDA(ctx, F.lightCdf.reserve(std::max<size_t>(1, em.size()) * 4));
  NOMAD_CUDA(ctx, F.lightPdf.reserve((size_t)P * 4));
  NOMAD_CUDA(ctx, F.lightMeta.reserve(sizeof(LightMeta)));
  NOMAD_CUDA(ctx, cudaMemset(F.lightPdf.p, 0, (size_t)P * 4));
  // hit-probability posterior: Beta(1, 1), probability 0.5, variance 1/12, mass 2
  NOMAD_CUDA(ctx, R.tlas.reserve(std::max<size_t>(1, R.hostTlas.size()) * 4));
  if (!R.hostTlas.empty())
    NOMAD_CUDA(ctx, cudaMemcpy(R.tlas.p, R.hostTlas.data(), R.hostTlas.size() * 4, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, R.tests.reserve((size_t)N * 4));
  NOMAD_CUDA(ctx, cudaMemset(R.tests.p, 0, (size_t)N * 4));
  NOMAD_CUDA(ctx, R.post.reserve((size_t)N * kPostWords * 4));
  {
    std::vector<float> post((size_t)N * kPostWords, 0.0f);
    for (uint32_t o = 0; o < N; ++o) {
      float *q = post.data() + (size_t)o * kPostWords;
      q[0] = 1.0f;
      q[1] = 1.0f;
      q[2] = 0.5f;
      q[3] = 1.0f / 12.0f;
      q[4] = 2.0f;
    }
    NOMAD_CUDA(ctx, cudaMemcpy(R.post.p, post.data(), post.size() * 4, cudaMemcpyHostToDevice));
  }
  R.testsOn = false;
  R.probOn = false;
  R.probOrder.clear();
  R.prevSegments = R.prevEscapes = 0;
  R.lastToggle.clear();
  R.energyHist.clear();
  R.energyTotal.clear();
  R.energyEmit.clear();
  R.frame = 0;
  R.havePrevCam = false;
  R.ready = true;
  F.lightsDirty = true;
  return nomad_residency_mirror(ctx);
}

// Copies the host residency state (after upload or a host-side flush) to the device arrays.
nomad_status nomad_residency_mirror(nomad_ctx *ctx) {
  auto &R = ctx->res;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(R.objRes.p, ctx->objResident.data(), ctx->objectCount, cudaMemcpyHostToDevice,
                                  ctx->stream));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(R.primAct.p, ctx->primActive.data(), ctx->primCount, cudaMemcpyHostToDevice,
                                  ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  ctx->frame.lightsDirty = true;
  return NOMAD_OK;
}

nomad_status nomad_lights_update(nomad_ctx *ctx) {
  FrameState &F = ctx->frame;
  if (!F.lightsDirty) return NOMAD_OK;
  auto &R = ctx->res;
  k_lights_rebuild<<<1, 1024, 0, ctx->stream>>>(R.emissive.as<const uint4>(), R.emissiveCount,
                                                R.primAct.as<const uint8_t>(), R.objRes.as<const uint8_t>(),
                                                F.lightIdx.as<uint32_t>(), F.lightCdf.as<float>(), F.lightPdf.as<float>(),
                                                F.lightMeta.as<LightMeta>(), ctx->prims.as<const float4>(),
                                                ctx->materials.as<const float4>(), F.lightRec.as<float4>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  F.lightsDirty = false;
  return NOMAD_OK;
}

namespace {

float clamp_unit(float v) { return std::min(std::max(v, 0.0f), 1.0f); }

// Bounding sphere of every primitive (Renderer.cpp:3158-3173): spheres as they are; triangles
// around the centroid, radius the farthest vertex; rectangles around the centre, radius |u| + |v|.
void prim_spheres(const nomad_ctx *ctx, std::vector<float> &out) {
  const uint32_t P = ctx->primCount;
  out.assign((size_t)P * 4, 0.0f);
  auto len = [](float x, float y, float z) { return std::sqrt(x * x + y * y + z * z); };
  for (uint32_t i = 0; i < P; ++i) {
    const float *g = ctx->hostPrims.data() + 28ull * i;
    const int type = (int)g[3];
    float *o = out.data() + 4ull * i;
    if (type == 0) {
      o[0] = g[0]; o[1] = g[1]; o[2] = g[2]; o[3] = g[4];
    } else if (type == 1) {
      const float cx = (g[0] + g[4] + g[8]) / 3.0f, cy = (g[1] + g[5] + g[9]) / 3.0f,
                  cz = (g[2] + g[6] + g[10]) / 3.0f;
      float r = len(g[0] - cx, g[1] - cy, g[2] - cz);
      r = std::max(r, len(g[4] - cx, g[5] - cy, g[6] - cz));
      r = std::max(r, len(g[8] - cx, g[9] - cy, g[10] - cz));
      o[0] = cx; o[1] = cy; o[2] = cz; o[3] = r;
    } else {
      o[0] = g[0]; o[1] = g[1]; o[2] = g[2];
      o[3] = len(g[4], g[5], g[6]) + len(g[8], g[9], g[10]);
    }
  }
}

// Camera of a view for the angular frustum test (Renderer::isInView, Renderer.cpp:1765-1817).
struct AngleCam {
  float pos[3], fwd[3], right[3], up[3];
  float halfV, halfH;  // vertical and horizontal half field of view (radians)
  bool fwdValid;
};

AngleCam angle_cam(const nomad_view &v) {
  AngleCam c{};
  float U[3], V[3], f[3];
  for (int k = 0; k < 3; ++k) {
    c.pos[k] = v.camera_pos[k];
    U[k] = v.viewport_u[k];
    V[k] = v.viewport_v[k];
    f[k] = v.first_pixel[k] + 0.5f * U[k] + 0.5f * V[k] - c.pos[k];
  }
  const float fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (int k = 0; k < 3; ++k) c.fwd[k] = f[k] / fl;
  const float fl2 = c.fwd[0] * c.fwd[0] + c.fwd[1] * c.fwd[1] + c.fwd[2] * c.fwd[2];
  c.fwdValid = fl2 >= 1e-6f;
  // camera up: opposite of the viewport's v axis (rows run downwards)
  float up[3] = {-V[0], -V[1], -V[2]};
  float ul2 = up[0] * up[0] + up[1] * up[1] + up[2] * up[2];
  if (ul2 < 1e-6f) {
    up[0] = 0.0f; up[1] = 1.0f; up[2] = 0.0f;
    ul2 = 1.0f;
  }
  const float ul = std::sqrt(ul2);
  for (int k = 0; k < 3; ++k) up[k] /= ul;
  float r[3] = {c.fwd[1] * up[2] - c.fwd[2] * up[1], c.fwd[2] * up[0] - c.fwd[0] * up[2],
                c.fwd[0] * up[1] - c.fwd[1] * up[0]};
  float rl2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  if (rl2 < 1e-6f) {
    r[0] = 1.0f; r[1] = 0.0f; r[2] = 0.0f;
    rl2 = 1.0f;
  }
  const float rl = std::sqrt(rl2);
  for (int k = 0; k < 3; ++k) c.right[k] = r[k] / rl;
  float u2[3] = {c.right[1] * c.fwd[2] - c.right[2] * c.fwd[1], c.right[2] * c.fwd[0] - c.right[0] * c.fwd[2],
                 c.right[0] * c.fwd[1] - c.right[1] * c.fwd[0]};
  const float u2l = std::sqrt(u2[0] * u2[0] + u2[1] * u2[1] + u2[2] * u2[2]);
  for (int k = 0; k < 3; ++k) c.up[k] = u2[k] / u2l;
  // vertical half angle from the viewport height at unit distance; aspect from the pixel counts
  const float vl = std::sqrt(V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
  c.halfV = std::atan(0.5f * vl / fl);
  if (c.halfV <= 0.0f) c.halfV = 1e-3f;
  const float aspect = v.height > 0 ? (float)v.width / (float)v.height : 1.0f;
  c.halfH = std::atan(std::tan(c.halfV) * aspect);
  return c;
}

bool in_view(const AngleCam &c, const float *sph) {
  const float tx = sph[0] - c.pos[0], ty = sph[1] - c.pos[1], tz = sph[2] - c.pos[2];
  const float dist = std::sqrt(tx * tx + ty * ty + tz * tz);
  if (dist < 1e-5f) return true;
  if (!c.fwdValid) return true;
  const float dx = tx / dist, dy = ty / dist, dz = tz / dist;
  const float fd = dx * c.fwd[0] + dy * c.fwd[1] + dz * c.fwd[2];
  if (fd <= 0.0f) return false;
  const float ra = std::asin(std::min(sph[3] / dist, 1.0f));
  const float h = std::atan2(std::fabs(dx * c.right[0] + dy * c.right[1] + dz * c.right[2]), fd);
  const float vv = std::atan2(std::fabs(dx * c.up[0] + dy * c.up[1] + dz * c.up[2]), fd);
  return h <= c.halfH + ra && vv <= c.halfV + ra;
}

float sanitize(float v) {
  const float fmax = std::numeric_limits<float>::max();
  if (std::isnan(v)) return -fmax;
  if (v >= fmax) return fmax;
  if (v <= -fmax) return -fmax;
  return v;
}

// updateRayHitBudget per primitive (RendererResidency.cpp:2755-2964) with the cooldown decrement
// of updateResidency (:205-207) and the counter pass of processRayHitCounters.
nomad_status rayhit_prim_step(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view &view,
                              uint32_t *toggled) {
  auto &R = ctx->res;
  const uint32_t P = ctx->primCount;
  if (!toggled) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the per-primitive policy runs synchronously");
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (!R.primHitsOn) {
    NOMAD_CUDA(ctx, R.primHits.reserve((size_t)P * 4));
    NOMAD_CUDA(ctx, cudaMemsetAsync(R.primHits.p, 0, (size_t)P * 4, ctx->stream));
    R.primHitsHost.assign(P, 0);
    R.primCooldown.assign(P, 0);
    R.primScore.assign(P, 0.0f);
    R.primVisible.assign(P, 0);
    prim_spheres(ctx, R.primSphere);
    R.primRebuild = 0;
    R.primHitsOn = true;
    ctx->frame.clearGraphs();  // the shading kernel now also counts per primitive
  }
  // counters -> decayed scores
  NOMAD_CUDA(ctx, cudaMemcpyAsync(R.primHitsHost.data(), R.primHits.p, (size_t)P * 4, cudaMemcpyDeviceToHost,
                                  ctx->stream));
  NOMAD_CUDA(ctx, cudaMemsetAsync(R.primHits.p, 0, (size_t)P * 4, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  for (uint32_t i = 0; i < P; ++i) R.primScore[i] = R.primScore[i] * prm->hit_decay + (float)R.primHitsHost[i];
  ++R.primStep;  // every primitive cooldown counts down by one
  *toggled = 0;
  if (R.primRebuild > 0) {
    --R.primRebuild;
    return NOMAD_OK;
  }
  const float motion = clamp_unit(prm->camera_motion), pressure = clamp_unit(prm->memory_pressure);
  const float frac = std::min(std::max(prm->target_fraction + 0.10f * motion - 0.24f * pressure, 0.34f), 0.92f);
  const bool unlimited = prm->max_toggles == 0;
  const size_t budget = std::max<size_t>(
      1, (size_t)std::llround((double)std::max<uint32_t>(prm->max_toggles, 1) *
                              (1.0 + 0.45 * (double)motion + 0.60 * (double)pressure)));
  const AngleCam cam = angle_cam(view);
  const float keep = 0.5f + (0.2f - 0.5f) * pressure;  // lerpFloat(0.5, 0.2, pressure)
  std::vector<float> adj(P);
  for (uint32_t i = 0; i < P; ++i) {
    const bool vis = in_view(cam, R.primSphere.data() + 4ull * i);
    R.primVisible[i] = vis ? 1 : 0;
    float sc = R.primScore[i];
    if (!vis) {
      if (R.primHitsHost[i] == 0) sc = 0.0f;
      else sc *= keep;
    } else if (sc <= 0.0f) {
      sc = 1.0f;
    }
    adj[i] = sanitize(sc);
  }
  const size_t minActive = std::min<size_t>(P, prm->min_active);
  size_t target = (size_t)std::ceil((float)P * frac);
  target = std::min<size_t>(std::max(target, minActive), P);
  // every index in (score desc, index asc) order: the reference's partial_sort prefix, extended
  // with the same order past it
  std::vector<uint32_t> order(P);
  for (uint32_t i = 0; i < P; ++i) order[i] = i;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    if (adj[a] == adj[b]) return a < b;
    return adj[a] > adj[b];
  });
  std::vector<uint8_t> desired(P, 0);
  for (size_t k = 0; k < target; ++k) desired[order[k]] = 1;
  const size_t reserve = std::min<size_t>(P, (size_t)std::ceil((float)P * (0.02f + 0.06f * motion)));
  size_t promoted = 0;
  for (uint32_t idx : order) {
    if (promoted >= reserve) break;
    if (!R.primVisible[idx]) continue;
    desired[idx] = 1;
    ++promoted;
  }
  for (size_t k = 0; k < minActive; ++k) desired[order[k]] = 1;
  uint32_t toggles = 0;
  for (uint32_t i = 0; i < P; ++i) {
    const bool want = desired[i] != 0;
    if (want == (ctx->primActive[i] != 0)) continue;
    if (!unlimited) {
      if (R.primCooldown[i] > R.primStep) continue;
      if (toggles >= budget) break;
    }
    int32_t changed = 0;
    nomad_status st = nomad_residency_set_primitive_active(ctx, i, want ? 1 : 0, &changed);
    if (st != NOMAD_OK) return st;
    if (changed) {
      R.primCooldown[i] = R.primStep + prm->state_cooldown;
      ++toggles;
    }
  }
  bool any = false;
  for (uint32_t i = 0; i < P && !any; ++i) any = ctx->primActive[i] != 0;
  if (!any && P > 0) {
    int32_t changed = 0;
    nomad_status st = nomad_residency_set_primitive_active(ctx, order[0], 1, &changed);
    if (st != NOMAD_OK) return st;
    if (changed) {
      R.primCooldown[order[0]] = R.primStep + prm->state_cooldown;
      ++toggles;
    }
  }
  if (toggles) {
    R.primRebuild = prm->rebuild_cooldown;
    nomad_status st = nomad_residency_flush(ctx);
    if (st != NOMAD_OK) return st;
  }
  *toggled = toggles;
  return NOMAD_OK;
}

// Bounding sphere of object o from its BLAS root box (Renderer.cpp:3272-3278: centre of the box,
// radius to its max corner); false for an object without primitives.
bool object_sphere(const nomad_ctx *ctx, uint32_t o, float *sph) {
  const nomad::TraversalLayout &L = ctx->layout;
  const float *mn, *mx;
  const int64_t slot = L.objSlot[o];
  if (slot >= 0) {
    const float *p = L.pnodes.data() + 16ull * (uint64_t)(slot / 2);
    mn = (slot & 1) ? p + 8 : p;
    mx = (slot & 1) ? p + 12 : p + 4;
  } else if (slot == -1) {
    mn = L.rootMin;
    mx = L.rootMax;
  } else {
    return false;
  }
  float c[3];
  for (int k = 0; k < 3; ++k) c[k] = (mn[k] + mx[k]) * 0.5f;
  const float dx = mx[0] - c[0], dy = mx[1] - c[1], dz = mx[2] - c[2];
  sph[0] = c[0];
  sph[1] = c[1];
  sph[2] = c[2];
  sph[3] = std::sqrt(dx * dx + dy * dy + dz * dz);
  return true;
}

// updateLODByDistance (RendererResidency.cpp:759-964) with the per-frame cooldown decrement of
// updateResidency (:208-210) and setObjectActive's cooldown (:1025).
nomad_status distance_lod_step(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view &view,
                               uint32_t *toggled) {
  auto &R = ctx->res;
  const uint32_t N = ctx->objectCount;
  if (!toggled) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the DistanceLOD policy runs synchronously");
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (!R.lodOn) {
    R.objCooldown.assign(N, 0);
    R.lodDist.assign(N, 0.0f);
    R.lodFlags.assign(N, 0);
    R.lodOn = true;
  }
  for (uint32_t &c : R.objCooldown)
    if (c > 0) --c;
  const float motion = clamp_unit(prm->camera_motion), pressure = clamp_unit(prm->memory_pressure);
  const size_t budget = std::max<size_t>(
      1, (size_t)std::llround((double)std::max<uint32_t>(prm->max_toggles, 1) *
                              (1.0 + 0.40 * (double)motion + 0.60 * (double)pressure)));
  const AngleCam cam = angle_cam(view);
  constexpr float kDegToRad = 0.0174532925199432957692f;
  const float enterMargin = std::max(prm->lod_enter_view_degrees, 0.0f) * kDegToRad;
  const float exitMargin = std::max(std::max(prm->lod_exit_view_degrees, 0.0f) * kDegToRad, enterMargin);
  const float fmax = std::numeric_limits<float>::max();
  std::vector<uint32_t> order(N);
  for (uint32_t o = 0; o < N; ++o) {
    order[o] = o;
    float sph[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    object_sphere(ctx, o, sph);
    const float tx = sph[0] - cam.pos[0], ty = sph[1] - cam.pos[1], tz = sph[2] - cam.pos[2];
    const float dtc = std::sqrt(tx * tx + ty * ty + tz * tz);
    const float dist = dtc - sph[3];
    const float fd = cam.fwdValid ? tx * cam.fwd[0] + ty * cam.fwd[1] + tz * cam.fwd[2] : 0.0f;
    const bool behind = cam.fwdValid && fd + sph[3] <= 0.0f;
    R.lodDist[o] = behind ? fmax : std::max(dist, 0.0f);
    bool enter = true, exit = true;
    if (cam.fwdValid) {
      if (dtc <= 1e-5f || behind) {
        enter = exit = !behind;
      } else {
        const float depth = std::max(fd, 1e-5f);
        const float horiz = tx * cam.right[0] + ty * cam.right[1] + tz * cam.right[2];
        const float vert = tx * cam.up[0] + ty * cam.up[1] + tz * cam.up[2];
        const float ha = std::atan2(std::fabs(horiz), depth), va = std::atan2(std::fabs(vert), depth);
        const float ra = std::asin(std::min(sph[3] / dtc, 1.0f));
        enter = ha <= cam.halfH + ra + enterMargin && va <= cam.halfV + ra + enterMargin;
        exit = ha <= cam.halfH + ra + exitMargin && va <= cam.halfV + ra + exitMargin;
      }
    }
    R.lodFlags[o] = (uint8_t)((enter ? 1 : 0) | (exit ? 2 : 0) | (behind ? 4 : 0));
  }
  // nearest first; equal distances by object index
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    if (R.lodDist[a] == R.lodDist[b]) return a < b;
    return R.lodDist[a] < R.lodDist[b];
  });
  uint32_t toggles = 0;
  for (uint32_t o : order) {
    const nomad_instance_record &ir = ctx->instances[o];
    const uint32_t count = ir.primitive_count, activeCount = ctx->objActiveCount[o];
    const bool active = activeCount > 0;
    const bool view_ok = active ? (R.lodFlags[o] & 2) != 0 : (R.lodFlags[o] & 1) != 0;
    const bool behind = (R.lodFlags[o] & 4) != 0;
    const float d = R.lodDist[o];
    const bool want = view_ok && !behind && (active ? d <= prm->lod_exit_distance : d < prm->lod_enter_distance);
    if (R.objCooldown[o] != 0 || want == active) continue;
    const uint32_t needed = want ? count - activeCount : activeCount;
    if (needed == 0) continue;
    if ((size_t)toggles + 1 > budget) continue;
    uint32_t n = 0;
    nomad_status st = nomad_residency_set_object_active(ctx, o, want ? 1 : 0, &n);
    if (st != NOMAD_OK) return st;
    const bool fullyInactive = ctx->objActiveCount[o] == 0;
    const bool nowActive = ctx->objActiveCount[o] > 0;
    if (n > 0 || nowActive != active || fullyInactive) R.objCooldown[o] = prm->state_cooldown;
    if (n > 0) ++toggles;
  }
  bool any = false;
  for (uint32_t o = 0; o < N && !any; ++o) any = ctx->objActiveCount[o] > 0;
  if (!any && ctx->primCount > 0) {
    int32_t changed = 0;
    nomad_status st = nomad_residency_set_primitive_active(ctx, 0, 1, &changed);
    if (st != NOMAD_OK) return st;
  }
  nomad_status st = nomad_residency_flush(ctx);
  if (st != NOMAD_OK) return st;
  *toggled = toggles;
  return NOMAD_OK;
}

// objectCoverageForSphere (RendererResidency.cpp:4130-4182) of every object's bounding sphere:
// the projected disc's pixel area times the cosine to the view axis, at most the screen, 0 outside
// the angular frustum (isInView), behind the camera or well outside horizontally. inView receives
// the frustum test of each sphere.
void object_coverage(const nomad_ctx *ctx, const nomad_view &view, std::vector<float> &cov,
                     std::vector<uint8_t> &inView) {
  const uint32_t N = ctx->objectCount;
  cov.assign(N, 0.0f);
  inView.assign(N, 0);
  const float W = (float)view.width, H = (float)view.height;
  float screenArea = W * H;
  if (screenArea <= 0.0f) screenArea = 1.0f;
  const AngleCam cam = angle_cam(view);
  // the camera's own up, not re-orthogonalised
  float tanHalf = std::tan(cam.halfV);
  if (tanHalf <= 0.0f) tanHalf = 1e-3f;
  float V[3], upRaw[3];
  for (int k = 0; k < 3; ++k) {
    V[k] = view.viewport_v[k];
    upRaw[k] = -V[k];
  }
  const float ul = std::sqrt(upRaw[0] * upRaw[0] + upRaw[1] * upRaw[1] + upRaw[2] * upRaw[2]);
  for (int k = 0; k < 3; ++k) upRaw[k] /= ul;
  float right[3] = {cam.fwd[1] * upRaw[2] - cam.fwd[2] * upRaw[1], cam.fwd[2] * upRaw[0] - cam.fwd[0] * upRaw[2],
                    cam.fwd[0] * upRaw[1] - cam.fwd[1] * upRaw[0]};
  const float rl2 = right[0] * right[0] + right[1] * right[1] + right[2] * right[2];
  if (rl2 < 1e-6f) {
    right[0] = 1.0f; right[1] = 0.0f; right[2] = 0.0f;
  } else {
    const float rl = std::sqrt(rl2);
    for (int k = 0; k < 3; ++k) right[k] /= rl;
  }
  const float aspect = H > 0.0f ? W / H : 1.0f;
  const float hHalf = std::atan(tanHalf * aspect);
  constexpr float kPi = 3.14159265358979323846f;
  for (uint32_t o = 0; o < N; ++o) {
    float sph[4];
    if (!object_sphere(ctx, o, sph)) continue;
    if (!in_view(cam, sph)) continue;
    inView[o] = 1;
    const float tx = sph[0] - cam.pos[0], ty = sph[1] - cam.pos[1], tz = sph[2] - cam.pos[2];
    const float depth = tx * cam.fwd[0] + ty * cam.fwd[1] + tz * cam.fwd[2];
    if (depth <= 1e-3f) continue;
    const float dist = std::sqrt(tx * tx + ty * ty + tz * tz);
    const float cosAngle = depth / std::max(dist, 1e-3f);
    const float horiz = tx * right[0] + ty * right[1] + tz * right[2];
    if (std::atan2(std::fabs(horiz), depth) > hHalf + 0.1f) continue;
    float rp = (sph[3] / depth) / tanHalf * (H * 0.5f);
    rp = std::max(rp, 0.0f);
    const float area = kPi * rp * rp;
    cov[o] = std::min(area * std::max(cosAngle, 0.0f), screenArea);
  }
}

// updateScreenSpaceFootprint (RendererResidency.cpp:4092-4396), one mesh group per object.
nomad_status screen_space_step(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view &view,
                               uint32_t *toggled) {
  auto &R = ctx->res;
  const uint32_t N = ctx->objectCount, P = ctx->primCount;
  if (!toggled) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the ScreenSpace policy runs synchronously");
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (!R.lodOn) {
    R.objCooldown.assign(N, 0);
    R.lodDist.assign(N, 0.0f);
    R.lodFlags.assign(N, 0);
    R.lodOn = true;
  }
  if (R.primCooldown.size() != P) R.primCooldown.assign(P, 0);
  for (uint32_t &c : R.objCooldown)
    if (c > 0) --c;
  ++R.primStep;  // every primitive cooldown counts down by one
  const float motion = clamp_unit(prm->camera_motion), pressure = clamp_unit(prm->memory_pressure);
  const float frac = std::min(std::max(prm->target_fraction + 0.08f * motion - 0.10f * pressure, 0.50f), 0.94f);
  const size_t budget = std::max<size_t>(
      1, (size_t)std::llround((double)std::max<uint32_t>(prm->max_toggles, 1) *
                              (1.0 + 0.40 * (double)motion + 0.50 * (double)pressure)));
  const float W = (float)view.width, H = (float)view.height;
  float screenArea = W * H;
  if (screenArea <= 0.0f) screenArea = 1.0f;
  std::vector<float> cov;
  std::vector<uint8_t> inView;
  object_coverage(ctx, view, cov, inView);
  std::vector<uint32_t> order(N);
  for (uint32_t o = 0; o < N; ++o) order[o] = o;
  for (uint32_t o = 0; o < N; ++o) R.lodDist[o] = cov[o];
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const float ca = sanitize(cov[a]), cb = sanitize(cov[b]);
    if (ca == cb) return a < b;
    return ca > cb;
  });
  const size_t minActive = std::min<size_t>(P, prm->min_active);
  const float target = screenArea * frac;
  std::vector<uint8_t> desired(N, 0);
  size_t enabled = 0;
  float acc = 0.0f;
  for (uint32_t g : order) {
    const size_t count = ctx->instances[g].primitive_count;
    if (count == 0) continue;
    const float c = cov[g];
    const bool minSat = enabled >= minActive, covSat = acc >= target;
    if (minSat && covSat) break;
    if (minSat && c < prm->min_pixel_coverage) continue;
    if (minSat && c <= 0.0f) continue;
    desired[g] = 1;
    enabled += count;
    acc += c;
  }
  for (uint32_t g : order) {
    if (enabled >= minActive) break;
    const size_t count = ctx->instances[g].primitive_count;
    if (desired[g] || count == 0) continue;
    desired[g] = 1;
    enabled += count;
    acc += cov[g];
  }
  size_t toggledPrims = 0;
  for (uint32_t g : order) {
    if (toggledPrims >= budget) break;
    const bool want = desired[g] != 0, active = ctx->objActiveCount[g] > 0;
    if (want == active) continue;
    if (R.objCooldown[g] > 0) continue;
    const nomad_instance_record &ir = ctx->instances[g];
    bool blocked = false;
    for (uint32_t p = ir.primitive_base; p < ir.primitive_base + ir.primitive_count && !blocked; ++p)
      if ((ctx->primActive[p] != 0) != want && R.primCooldown[p] > R.primStep) blocked = true;
    if (blocked) continue;
    for (uint32_t p = ir.primitive_base; p < ir.primitive_base + ir.primitive_count; ++p)
      if ((ctx->primActive[p] != 0) != want) R.primCooldown[p] = R.primStep + prm->state_cooldown;
    uint32_t n = 0;
    nomad_status st = nomad_residency_set_object_active(ctx, g, want ? 1 : 0, &n);
    if (st != NOMAD_OK) return st;
    if (n > 0 || (ctx->objActiveCount[g] > 0) != active || ctx->objActiveCount[g] == 0)
      R.objCooldown[g] = prm->state_cooldown;
    if (n > 0) toggledPrims = std::min(toggledPrims + n, budget);
  }
  bool any = false;
  for (uint32_t o = 0; o < N && !any; ++o) any = ctx->objActiveCount[o] > 0;
  if (!any) {
    size_t fallback = 0;
    for (uint32_t g : order) {
      const size_t count = ctx->instances[g].primitive_count;
      if (count == 0) continue;
      uint32_t n = 0;
      nomad_status st = nomad_residency_set_object_active(ctx, g, 1, &n);
      if (st != NOMAD_OK) return st;
      if (n > 0) {
        R.objCooldown[g] = prm->state_cooldown;
        fallback += count;
        any = true;
      }
      if (any && fallback >= minActive) break;
    }
  }
  nomad_status st = nomad_residency_flush(ctx);
  if (st != NOMAD_OK) return st;
  *toggled = (uint32_t)toggledPrims;
  return NOMAD_OK;
}

}  // namespace

extern "C" nomad_status nomad_residency_posterior(nomad_ctx *ctx, float *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady || !ctx->res.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  NOMAD_DEVICE_SCOPE(ctx);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(out, ctx->res.post.p, (size_t)ctx->objectCount * kPostWords * 4,
                                  cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_count_tests(nomad_ctx *ctx, int32_t on, uint32_t *tests) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady || !ctx->res.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  NOMAD_DEVICE_SCOPE(ctx);
  auto &R = ctx->res;
  if (tests) {
    NOMAD_CUDA(ctx, cudaMemcpyAsync(tests, R.tests.p, (size_t)ctx->objectCount * 4, cudaMemcpyDeviceToHost,
                                    ctx->stream));
    NOMAD_CUDA(ctx, cudaMemsetAsync(R.tests.p, 0, (size_t)ctx->objectCount * 4, ctx->stream));
    NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if ((on != 0) != R.testsOn) {
    R.testsOn = on != 0;
    ctx->frame.clearGraphs();
  }
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_fallback_steps(nomad_ctx *ctx, uint64_t *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  *out = ctx->res.fallbackSteps;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_object_state(nomad_ctx *ctx, float *distance, uint8_t *flags,
                                                     uint32_t *cooldowns) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  auto &R = ctx->res;
  if (!R.lodOn) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "the DistanceLOD policy has not run");
  const size_t N = ctx->objectCount;
  if (distance) std::memcpy(distance, R.lodDist.data(), N * 4);
  if (flags) std::memcpy(flags, R.lodFlags.data(), N);
  if (cooldowns) std::memcpy(cooldowns, R.objCooldown.data(), N * 4);
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_prim_state(nomad_ctx *ctx, uint32_t *hits, float *scores, uint32_t *cooldowns,
                                                   uint8_t *visible, uint8_t *active) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  auto &R = ctx->res;
  if (!R.primHitsOn) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "the per-primitive policy has not run");
  const size_t P = ctx->primCount;
  if (hits) {
    NOMAD_CUDA(ctx, cudaMemcpyAsync(hits, R.primHits.p, P * 4, cudaMemcpyDeviceToHost, ctx->stream));
    NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  if (scores) std::memcpy(scores, R.primScore.data(), P * 4);
  if (cooldowns)
    for (size_t i = 0; i < P; ++i) cooldowns[i] = R.primCooldown[i] > R.primStep ? R.primCooldown[i] - R.primStep : 0u;
  if (visible) std::memcpy(visible, R.primVisible.data(), P);
  if (active) {
    nomad_status hs = nomad_residency_sync_host(ctx);
    if (hs != NOMAD_OK) return hs;
    std::memcpy(active, ctx->primActive.data(), P);
  }
  return NOMAD_OK;
}

namespace {

// The per-object pass of a residency step on the context's stream: camera frame, features and
// keys (the learned scorer's or the ray-hit key), then the hit-probability posterior and the
// ray-hit prior. Counting of rays tested starts with the first step that asks for it.
nomad_status object_pass(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view *camera) {
  const uint32_t N = ctx->objectCount;
  auto &R = ctx->res;
  cudaStream_t s = ctx->stream;
  // camera frame from the view (populateViewportUniforms: first_pixel = pos - w - U/2 - V/2)
  CamDev cam;
  float c[3], U[3], V[3];
  for (int k = 0; k < 3; ++k) {
    cam.pos[k] = camera->camera_pos[k];
    U[k] = camera->viewport_u[k];
    V[k] = camera->viewport_v[k];
    c[k] = camera->first_pixel[k] + 0.5f * U[k] + 0.5f * V[k] - cam.pos[k];
  }
  auto nrm = [](const float *a, float *o) {
    float l = std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    for (int k = 0; k < 3; ++k) o[k] = a[k] / l;
    return l;
  };
  float dl = nrm(c, cam.fwd);
  float ul = nrm(U, cam.right);
  float vl = nrm(V, cam.up);
  for (int k = 0; k < 3; ++k) cam.up[k] = -cam.up[k];
  cam.halfW = 0.5f * ul / dl;
  cam.halfH = 0.5f * vl / dl;
  cam.speed = 0.0f;
  if (R.havePrevCam) {
    float d0 = cam.pos[0] - R.prevCam[0], d1 = cam.pos[1] - R.prevCam[1], d2 = cam.pos[2] - R.prevCam[2];
    cam.speed = std::sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  }
  for (int k = 0; k < 3; ++k) R.prevCam[k] = cam.pos[k];
  R.havePrevCam = true;
  FeatArgs fa{N, cam, R.bounds.as<const float4>(), R.bytes.as<const unsigned long long>(), R.tris.as<const uint32_t>(),
              R.emit.as<const float>(), R.objRes.as<const uint8_t>(), ctx->objHits.as<uint32_t>(), R.hist.as<uint32_t>(),
              R.score.as<float>(), R.lastHit.as<uint32_t>(), R.prevDist.as<float>(), R.visible.as<uint8_t>(),
              R.features.as<float>(), R.misc.as<uint32_t>(), R.frame, prm->hit_decay, prm->memory_pressure};
  if (prm->policy == NOMAD_POLICY_LEARNED) {
    // features and scores in one kernel (the scorer's CTAs compute their rows' features)
    nomad_status st = nomad_mlp_score_objects(ctx, &fa, R.keys.as<float>());
    if (st != NOMAD_OK) return st;
  } else {
    k_features<<<(N + 127) / 128, 128, 0, s>>>(fa, R.keys.as<float>());
    NOMAD_CUDA(ctx, cudaGetLastError());
  }
  // the hit-probability posterior, and the ray-hit prior on the keys
  const float window = prm->probability_window;
  PostArgs pa{N, R.frame, R.hist.as<const uint32_t>(), R.tests.as<uint32_t>(), R.visible.as<const uint8_t>(),
              R.objRes.as<const uint8_t>(), R.post.as<float>(), prm->probability_decay, prm->hit_decay,
              std::max(window, 1.0e-3f), prm->probability_idle_decay, prm->probability_threshold,
              (window > 0.0f && std::isfinite(window)) ? 1 : 0, prm->probability_idle_frames,
              prm->policy == NOMAD_POLICY_RAYHIT_BUDGET ? R.keys.as<float>() : nullptr, prm->rayhit_prior_scale};
  k_posterior<<<(N + 127) / 128, 128, 0, s>>>(pa);
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

// updateProbabilisticResidency (RendererResidency.cpp:2966-4090), its object-level path
// (:3389-4090), over the device posterior of the same step. One object at a time: every
// primitive of an object toggles with it, so the primitive cooldowns the reference checks equal
// the object's, and the primitive counts are the objects' (contribution = max(count, 1)).
// Visibility is the device frustum test of the per-object pass; the reference's "became
// visible" test compares isInView with the flag processRayHitCounters set from the same camera
// earlier in the frame, so it never fires and is left out. setObjectActive's side effects on the
// policy (desired state, promotion / demotion frame, pending flag, cooldown; :965-1031) are
// applied where it toggles.
nomad_status probabilistic_step(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view &view,
                                uint32_t *toggled) {
  auto &R = ctx->res;
  const uint32_t N = ctx->objectCount;
  if (!toggled) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the Probabilistic policy runs synchronously");
  if (N > kMaxSelectObjects)
    return nomad_fail(ctx, NOMAD_ERR_LIMIT, "the residency policies support at most 16384 objects");
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (!R.testsOn) {
    R.testsOn = true;
    ctx->frame.clearGraphs();  // the frame now also counts rays tested per object
  }
  if (!R.probOn) {
    R.probDesired.assign(N, 0);
    R.probPending.assign(N, 0);
    R.probPromoted.assign(N, 0);
    R.probDemoted.assign(N, 0);
    R.probDwell.assign(N, 0);
    R.probEvidence.assign(N, 0.0f);
    R.probOrder.resize(N);
    std::iota(R.probOrder.begin(), R.probOrder.end(), 0u);
    R.objCooldown.assign(N, 0);
    R.probOn = true;
  }
  for (uint32_t &c : R.objCooldown)
    if (c > 0) --c;
  cudaStream_t s = ctx->stream;
  nomad_status st = object_pass(ctx, prm, &view);
  if (st != NOMAD_OK) return st;
  const uint32_t frameNo = R.frame + 1;  // _renderedFrameCount: 0 means "never"
  ++R.frame;
  std::vector<float> post((size_t)N * kPostWords);
  std::vector<uint8_t> vis(N);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(post.data(), R.post.p, post.size() * 4, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(vis.data(), R.visible.p, N, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  auto P = [&](uint32_t o, int k) -> float & { return post[(size_t)o * kPostWords + k]; };
  auto testsLast = [&](uint32_t o) {
    uint32_t v;
    std::memcpy(&v, &post[(size_t)o * kPostWords + 8], 4);
    return v;
  };
  const size_t primCount = ctx->primCount;
  auto primitives = [&](uint32_t o) { return (size_t)std::max<uint32_t>(ctx->instances[o].primitive_count, 1u); };
  auto active = [&](uint32_t o) { return ctx->objActiveCount[o] > 0; };

  const float motion = clamp_unit(prm->camera_motion), pressure = clamp_unit(prm->memory_pressure);
  const float targetFraction =
      std::min(std::max(prm->target_fraction + 0.08f * motion - 0.12f * pressure, 0.45f), 0.93f);
  const size_t baseBudget = std::max<size_t>(prm->max_toggles, 1);
  const size_t toggleBudget = std::max<size_t>(
      1, (size_t)std::llround((double)baseBudget * (1.0 + 0.40 * (double)motion + 0.50 * (double)pressure)));
  constexpr float kPosteriorFloor = 1.0e-3f, kMinimalEvidence = 1.0e-3f, kEvidenceDecay = 0.9f, kSeed = 1.0f;
  const float window = prm->probability_window;
  const bool finiteWindow = window > 0.0f && std::isfinite(window);
  const float floorVisible = std::min(std::max(prm->visible_floor, 0.0f), 1.0f);
  const float scoringWindow = finiteWindow ? std::max(window, kPosteriorFloor) : std::max(64.0f, kPosteriorFloor);
  auto cl = [](float v) { return std::min(std::max(v, 0.0f), 1.0f); };
  auto evidence = [&](float mass, bool visible) {
    if (!(mass > 0.0f) || !std::isfinite(mass) || !visible) return 0.0f;
    return finiteWindow ? cl(mass / scoringWindow) : cl(mass / (mass + scoringWindow));
  };
  auto saneP = [&](float p) { return std::isfinite(p) ? cl(p) : 0.5f; };
  auto saneVar = [](float v) { return (!std::isfinite(v) || v < 0.0f) ? 0.0f : v; };
  auto regressedE = [&](float p, float e) {
    const float ce = cl(e);
    return saneP(p) * ce + 0.5f * (1.0f - ce);
  };
  auto scoreE = [&](float p, float var, float e) {
    return regressedE(p, e) + prm->uncertainty_boost * std::sqrt(std::max(saneVar(var), 0.0f));
  };
  auto score = [&](uint32_t o) { return scoreE(P(o, 2), P(o, 3), evidence(P(o, 4), vis[o] != 0)); };

  std::vector<uint8_t> desired = R.probDesired;
  auto &pending = R.probPending;
  const float threshold = prm->probability_threshold;
  const float hyst = std::min(std::max(prm->desired_hysteresis, 0.0f), 0.5f);
  const float enterT = cl(threshold + hyst), exitT = cl(threshold - hyst);
  const uint32_t dwellFrames = prm->demotion_dwell_frames;
  size_t desiredCount = 0;
  for (uint32_t i = 0; i < N; ++i) {
    const float prob = P(i, 2), var = P(i, 3), mass = P(i, 4);
    const bool visible = vis[i] != 0;
    const float rawE = evidence(mass, visible);
    const float buffered = std::max(cl(rawE), R.probEvidence[i] * kEvidenceDecay);
    R.probEvidence[i] = buffered;
    const float eff = regressedE(saneP(prob), buffered);
    const float boosted = scoreE(prob, var, buffered);
    const float enterScore = std::max(eff, boosted), exitScore = eff;
    const bool prev = desired[i] != 0;
    bool want = prev;
    const bool cooldownExpired = R.objCooldown[i] == 0;
    const bool lowEvidence = std::min(buffered, cl(rawE)) <= kMinimalEvidence;
    float promotion = enterScore, demotion = exitScore, evaluation = lowEvidence ? eff : enterScore;
    const bool dwellApplies = visible && dwellFrames > 0;
    if (!dwellApplies || demotion > exitT) R.probDwell[i] = 0;
    if (visible) {
      demotion = std::max(demotion, floorVisible);
      evaluation = std::max(evaluation, floorVisible);
    }
    if (promotion >= enterT) {
      want = true;
      R.probDwell[i] = 0;
    } else if (demotion <= exitT) {
      if (dwellApplies && prev) {
        if (R.probDwell[i] < dwellFrames) ++R.probDwell[i];
        want = R.probDwell[i] < dwellFrames;
      } else {
        want = false;
        R.probDwell[i] = 0;
      }
    } else if (cooldownExpired && !prev) {
      want = evaluation >= threshold;
      if (want) R.probDwell[i] = 0;
    }
    if (want && !prev) R.probPromoted[i] = frameNo;
    else if (!want && prev) R.probDemoted[i] = frameNo;
    desired[i] = want ? 1 : 0;
    if (!want) pending[i] = 0;
    if (want && !pending[i]) desiredCount += primitives(i);
  }
  const size_t minActive = std::min<size_t>(prm->min_active, primCount);
  auto &order = R.probOrder;
  std::vector<float> keys(N);
  for (uint32_t o = 0; o < N; ++o) keys[o] = sanitize(score(o));
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    if (keys[a] == keys[b]) return a < b;
    return keys[a] > keys[b];
  });
  size_t target = (size_t)std::ceil((float)primCount * targetFraction);
  target = std::max(target, minActive);
  if (target == 0 && primCount > 0) target = 1;
  target = std::min(target, primCount);
  auto trim = [&]() {
    if (target == 0 || desiredCount <= target) return;
    for (size_t pos = order.size(); pos-- > 0;) {
      if (desiredCount <= target) break;
      const uint32_t idx = order[pos];
      if (!desired[idx] || pending[idx]) continue;
      const size_t c = primitives(idx);
      desired[idx] = 0;
      pending[idx] = 0;
      R.probDemoted[idx] = frameNo;
      desiredCount = desiredCount > c ? desiredCount - c : 0;
    }
  };
  trim();
  std::vector<uint32_t> visibleExplore, hiddenExplore;
  for (uint32_t idx : order) {
    if (active(idx) || desired[idx]) continue;
    const float prob = P(idx, 2), mass = P(idx, 4);
    const bool visible = vis[idx] != 0;
    const float rawE = evidence(mass, visible);
    const float buffered = R.probEvidence[idx];
    const float eff = regressedE(prob, buffered);
    const bool lowEvidence = std::min(buffered, cl(rawE)) <= kMinimalEvidence;
    const float gated = (visible && lowEvidence) ? std::min(eff, threshold) : eff;
    if (gated > threshold) continue;
    const uint32_t rays = testsLast(idx);
    float ex = P(idx, 5);
    if (visible && (rays == 0 || lowEvidence)) ex = std::max(ex, kSeed);
    if (visible && rays > 0 && !lowEvidence) ex = std::max(ex, kPosteriorFloor);
    P(idx, 5) = ex;
    if (ex <= 0.0f) continue;
    (visible ? visibleExplore : hiddenExplore).push_back(idx);
  }
  auto exploreFirst = [&](uint32_t a, uint32_t b) {
    const float ea = sanitize(P(a, 5)), eb = sanitize(P(b, 5));
    if (ea == eb) {
      const uint32_t ra = testsLast(a), rb = testsLast(b);
      if (ra == rb) return a < b;
      return ra > rb;
    }
    return ea > eb;
  };
  std::sort(visibleExplore.begin(), visibleExplore.end(), exploreFirst);
  std::sort(hiddenExplore.begin(), hiddenExplore.end(), exploreFirst);
  auto recent = [&](uint32_t idx) {
    const uint32_t w = prm->recent_promotion_frames;
    if (w == 0) return false;
    const uint32_t last = std::max(R.probPromoted[idx], R.probDemoted[idx]);
    if (last == 0) return false;
    if (frameNo <= last) return true;
    return frameNo - last < w;
  };
  auto markDesired = [&](uint32_t idx) {
    desired[idx] = 1;
    R.probPromoted[idx] = frameNo;
    const size_t c = primitives(idx);
    if (!pending[idx]) desiredCount += c;
    if (vis[idx] && testsLast(idx) == 0 && P(idx, 5) < kSeed) P(idx, 5) = kSeed;
    return c;
  };
  auto promote = [&](const std::vector<uint32_t> &cands, size_t &slots, bool allowSuppressed) {
    if (slots == 0) return;
    for (uint32_t idx : cands) {
      if (slots == 0) break;
      if (desired[idx]) continue;
      if (!allowSuppressed && recent(idx)) continue;
      const size_t c = markDesired(idx);
      slots = slots <= c ? 0 : slots - c;
    }
  };
  auto remainingOf = [&](const std::vector<uint32_t> &cands) {
    size_t r = 0;
    for (uint32_t idx : cands)
      if (!desired[idx] && !pending[idx]) r += primitives(idx);
    return r;
  };
  if (desiredCount < minActive) {
    size_t slots = std::min(minActive - desiredCount, primCount > desiredCount ? primCount - desiredCount : 0);
    promote(visibleExplore, slots, false);
    promote(hiddenExplore, slots, false);
    if (slots > 0) {
      promote(visibleExplore, slots, true);
      promote(hiddenExplore, slots, true);
    }
  }
  if (desiredCount < minActive) {
    for (int allow = 0; allow < 2 && desiredCount < minActive; ++allow)
      for (uint32_t idx : order) {
        if (desiredCount >= minActive) break;
        if (desired[idx]) continue;
        if (!allow && recent(idx)) continue;
        markDesired(idx);
      }
  }
  const size_t remaining = remainingOf(visibleExplore) + remainingOf(hiddenExplore);
  if (remaining > 0 && desiredCount < primCount) {
    size_t slots = std::min({std::max<size_t>(1, minActive / 2), remaining, primCount - desiredCount});
    promote(visibleExplore, slots, false);
    promote(hiddenExplore, slots, false);
    if (slots > 0) {
      promote(visibleExplore, slots, true);
      promote(hiddenExplore, slots, true);
    }
  }
  desiredCount = 0;
  for (uint32_t idx = 0; idx < N; ++idx)
    if (desired[idx] && !pending[idx]) desiredCount += primitives(idx);
  trim();
  uint32_t fallback = N;
  if (!visibleExplore.empty()) fallback = visibleExplore.front();
  else if (!hiddenExplore.empty()) fallback = hiddenExplore.front();
  else if (!order.empty()) fallback = order.front();

  // setObjectActive with its side effects on the policy state
  auto setObject = [&](uint32_t o, bool want, uint32_t &n) -> nomad_status {
    const bool prevState = active(o);
    nomad_status r = nomad_residency_set_object_active(ctx, o, want ? 1 : 0, &n);
    if (r != NOMAD_OK) return r;
    const bool newState = active(o), fullyInactive = !newState;
    R.probDesired[o] = newState ? 1 : 0;
    if (newState) R.probPromoted[o] = frameNo;
    else R.probDemoted[o] = frameNo;
    if (!newState || n > 0) pending[o] = 0;
    if (n > 0 || prevState != newState || fullyInactive) R.objCooldown[o] = prm->state_cooldown;
    return NOMAD_OK;
  };
  std::vector<uint32_t> toggleOrder;
  std::vector<uint8_t> added(N, 0), appliedDesired(N, 0);
  auto append = [&](const std::vector<uint32_t> &cands) {
    for (uint32_t idx : cands)
      if (!added[idx]) {
        toggleOrder.push_back(idx);
        added[idx] = 1;
      }
  };
  std::vector<uint32_t> byPriority, pendingList;
  for (uint32_t idx : order)
    if (desired[idx]) byPriority.push_back(idx);
  for (uint32_t idx = 0; idx < N; ++idx)
    if (pending[idx]) pendingList.push_back(idx);
  append(pendingList);
  append(byPriority);
  append(visibleExplore);
  append(hiddenExplore);
  append(order);
  size_t toggledPrims = 0;
  const size_t maxToggles = toggleBudget;
  for (uint32_t idx : toggleOrder) {
    if (maxToggles == 0 || toggledPrims >= maxToggles) break;
    const bool want = desired[idx] != 0, current = active(idx);
    if (want == current) continue;
    if (R.objCooldown[idx] > 0) {
      if (want) pending[idx] = 1;
      continue;
    }
    const uint32_t count = ctx->instances[idx].primitive_count, activeCount = ctx->objActiveCount[idx];
    const size_t pendingToggles = want ? count - activeCount : activeCount;
    if (pendingToggles == 0) continue;
    const size_t remainingBudget = maxToggles > toggledPrims ? maxToggles - toggledPrims : 0;
    if (pendingToggles > remainingBudget) {
      if (want) pending[idx] = 1;
      continue;
    }
    uint32_t n = 0;
    st = setObject(idx, want, n);
    if (st != NOMAD_OK) return st;
    if (n > 0) {
      toggledPrims += std::min<size_t>(n, remainingBudget);
      if (want && !appliedDesired[idx]) {
        appliedDesired[idx] = 1;
        pending[idx] = 0;
        R.probDesired[idx] = 1;
      }
      if (!want) {
        P(idx, 5) = 0.0f;
        pending[idx] = 0;
        R.probDesired[idx] = 0;
      }
    }
  }
  bool anyActive = false;
  for (uint32_t o = 0; o < N && !anyActive; ++o) anyActive = active(o);
  if (!anyActive && N > 0) {
    const uint32_t fb = fallback < N ? fallback : 0u;
    const size_t remainingBudget = maxToggles > toggledPrims ? maxToggles - toggledPrims : 0;
    if (remainingBudget > 0) {
      uint32_t n = 0;
      st = setObject(fb, true, n);
      if (st != NOMAD_OK) return st;
      toggledPrims += std::min<size_t>(n, remainingBudget);
    }
    R.probDesired[fb] = 1;
    R.probPromoted[fb] = frameNo;
  }
  // the exploration scores the policy updated go back to the device posterior (one strided copy)
  NOMAD_CUDA(ctx, cudaMemcpy2DAsync(R.post.as<float>() + 5, kPostWords * 4, post.data() + 5, kPostWords * 4, 4, N,
                                    cudaMemcpyHostToDevice, s));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  st = nomad_residency_flush(ctx);
  if (st != NOMAD_OK) return st;
  *toggled = (uint32_t)toggledPrims;
  return NOMAD_OK;
}

// updateEnvironmentHitResidency (RendererResidency.cpp:4759-5155) and updatePredictiveResidency
// (:4397-4757), over the device posterior of the same step. Both rank objects by a weighted
// importance (EnvironmentHit: the hit probability, raised to an exploration prior for objects
// without evidence; Predictive: that times the ray-hit score per primitive), want objects in that
// order until the activation floor is reached and the mean escape probability of the wanted
// primitives is at most the escape threshold, then toggle with a budget that grows with the
// off-screen resident primitives and lets low-importance off-screen objects leave despite their
// cooldown. EnvironmentHit also moves the activation floor with the last frame's fraction of ray
// segments that escaped to the environment. Visibility is the device frustum test; no depth
// weights are configured (environmentDepthWeights empty: weight 1). setObjectActive's cooldown
// rule (:1025-1026) applies where an object toggles.
nomad_status environment_step(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view &view,
                              uint32_t *toggled, bool predictive) {
  auto &R = ctx->res;
  const uint32_t N = ctx->objectCount;
  if (!toggled) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the environment policies run synchronously");
  if (N > kMaxSelectObjects)
    return nomad_fail(ctx, NOMAD_ERR_LIMIT, "the residency policies support at most 16384 objects");
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (!R.testsOn) {
    R.testsOn = true;
    ctx->frame.clearGraphs();  // the frame now also counts rays tested per object
  }
  if (R.objCooldown.size() != N) R.objCooldown.assign(N, 0);
  if (R.probOrder.size() != N) {
    R.probOrder.resize(N);
    std::iota(R.probOrder.begin(), R.probOrder.end(), 0u);
  }
  for (uint32_t &c : R.objCooldown)
    if (c > 0) --c;
  cudaStream_t s = ctx->stream;
  nomad_status st = object_pass(ctx, prm, &view);
  if (st != NOMAD_OK) return st;
  ++R.frame;
  std::vector<float> post((size_t)N * kPostWords), score(N);
  std::vector<uint8_t> vis(N);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(post.data(), R.post.p, post.size() * 4, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(vis.data(), R.visible.p, N, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(score.data(), R.score.p, (size_t)N * 4, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  // the last frame's fraction of closest-hit segments that escaped (processRayHitCounters :8324-8328)
  uint64_t stats[4];
  st = nomad_render_stats(ctx, stats);
  if (st != NOMAD_OK) return st;
  if (stats[0] < R.prevSegments || stats[1] < R.prevEscapes) R.prevSegments = R.prevEscapes = 0;  // stats reset
  const uint64_t segments = stats[0] - R.prevSegments, escapes = stats[1] - R.prevEscapes;
  R.prevSegments = stats[0];
  R.prevEscapes = stats[1];
  const float globalEscape =
      segments > 0 ? (float)(uint32_t)escapes / (float)std::max<uint32_t>((uint32_t)segments, 1u) : 0.0f;

  auto Pf = [&](uint32_t o, int k) { return post[(size_t)o * kPostWords + k]; };
  auto testsLast = [&](uint32_t o) {
    uint32_t v;
    std::memcpy(&v, &post[(size_t)o * kPostWords + 8], 4);
    return v;
  };
  auto active = [&](uint32_t o) { return ctx->objActiveCount[o] > 0; };
  const size_t primCount = ctx->primCount;
  const float motion = clamp_unit(prm->camera_motion), pressure = clamp_unit(prm->memory_pressure);
  const float escapeThreshold =
      std::min(std::max(prm->env_escape_threshold + 0.03f * motion + 0.08f * pressure, 0.12f), 0.95f);
  const float targetFraction = std::min(std::max(prm->target_fraction + 0.08f * motion - 0.10f * pressure, 0.12f),
                                        predictive ? 0.92f : 0.94f);
  const size_t baseBudget = std::max<size_t>(prm->max_toggles, 1);
  const size_t toggleBudget = std::max<size_t>(
      1, (size_t)std::llround((double)baseBudget * (1.0 + 0.40 * (double)motion + 0.70 * (double)pressure)));
  constexpr float kPriorFloor = 1.0e-4f, kPriorScale = 0.5f, kVisibleBoost = 2.0f, kHiddenPenalty = 0.05f;
  constexpr float kSeed = 1.0f;  // kIdleVisibleExploreSeed
  std::vector<float> importance(N), weighted(N);
  for (uint32_t o = 0; o < N; ++o) {
    float prob = std::min(std::max(Pf(o, 2), 0.0f), 1.0f);
    const bool hasEvidence = testsLast(o) > 0, current = active(o), visible = vis[o] != 0;
    if (!hasEvidence && !current) {
      const float ex = std::max(Pf(o, 5), 0.0f);
      float prior = 1.0f - std::exp(-ex * kPriorScale);
      if (visible) prior = std::max(prior, 1.0f - std::exp(-kSeed * kPriorScale));
      prior = std::min(std::max(prior, kPriorFloor), 1.0f);
      prob = std::max(prob, prior);
    }
    importance[o] = prob;
    float sc = prob;
    if (predictive) {
      float hitScore = score[o];
      const uint32_t count = ctx->instances[o].primitive_count;
      if (count > 0) hitScore /= (float)count;
      if (hitScore <= 0.0f && (current || visible)) hitScore = 1.0f;
      sc = hitScore * prob;
    }
    const float depthWeight = 1.0f, visibilityWeight = visible ? kVisibleBoost : kHiddenPenalty;
    const float w = sc * std::max(depthWeight, 0.0f) * std::max(visibilityWeight, 0.0f);
    weighted[o] = std::isfinite(w) ? w : 0.0f;
  }
  auto &order = R.probOrder;
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    if (weighted[a] == weighted[b]) {
      if (importance[a] == importance[b]) return a < b;
      return importance[a] > importance[b];
    }
    return weighted[a] > weighted[b];
  });
  size_t minActive = std::min<size_t>(primCount, prm->min_active);
  if (minActive == 0 && primCount > 0) minActive = 1;
  size_t targetCount = 0;
  if (targetFraction > 0.0f && primCount > 0)
    targetCount = std::min((size_t)std::ceil(targetFraction * (float)primCount), primCount);
  size_t floorCount = std::max(minActive, targetCount);
  if (!predictive) {
    const float high = std::min(std::max(prm->env_high_escape, 0.0f), 1.0f);
    const float low = std::min(std::max(prm->env_low_escape, 0.0f), high);
    if (globalEscape > high) floorCount = std::min(primCount, (size_t)((float)floorCount * 1.5f));
    else if (globalEscape < low) floorCount = std::max(minActive, (size_t)((float)floorCount * 0.8f));
  }
  if (floorCount == 0 && primCount > 0) floorCount = 1;
  std::vector<uint8_t> desired(N, 0);
  size_t desiredCount = 0;
  float weightedEscape = 0.0f;
  auto averageEscape = [](size_t count, float w) { return count == 0 ? 1.0f : w / (float)count; };
  for (uint32_t idx : order) {
    const uint32_t count = ctx->instances[idx].primitive_count;
    if (count == 0) continue;
    if (!(desiredCount < floorCount) && !(averageEscape(desiredCount, weightedEscape) > escapeThreshold)) break;
    desired[idx] = 1;
    desiredCount += count;
    weightedEscape += (1.0f - importance[idx]) * (float)count;
  }
  if (desiredCount == 0 && primCount > 0)
    for (uint32_t idx : order) {
      const uint32_t count = ctx->instances[idx].primitive_count;
      if (count == 0) continue;
      desired[idx] = 1;
      desiredCount = count;
      weightedEscape = (1.0f - importance[idx]) * (float)count;
      break;
    }
  size_t offscreenActive = 0;
  for (uint32_t o = 0; o < N; ++o)
    if (active(o) && !vis[o]) offscreenActive += ctx->instances[o].primitive_count;
  size_t maxBudget = toggleBudget;
  if (offscreenActive > toggleBudget) maxBudget = std::max(toggleBudget, (offscreenActive + 1) / 2);
  const size_t reserved = maxBudget == 0 ? 0 : std::max<size_t>(1, maxBudget / 4);
  const size_t general = maxBudget > reserved ? maxBudget - reserved : 0;
  const size_t total = maxBudget + reserved;
  size_t toggledPrims = 0;
  auto setObject = [&](uint32_t o, bool want, uint32_t &n) -> nomad_status {
    const bool prevState = active(o);
    nomad_status r = nomad_residency_set_object_active(ctx, o, want ? 1 : 0, &n);
    if (r != NOMAD_OK) return r;
    const bool newState = active(o);
    if (n > 0 || prevState != newState || !newState) R.objCooldown[o] = prm->state_cooldown;
    return NOMAD_OK;
  };
  for (uint32_t idx : order) {
    const bool want = desired[idx] != 0, current = active(idx);
    if (want == current) continue;
    const bool visible = vis[idx] != 0;
    const bool bypass = current && !want && !visible && importance[idx] < escapeThreshold;
    if (!bypass && R.objCooldown[idx] > 0) continue;
    const uint32_t count = ctx->instances[idx].primitive_count;
    if (count == 0) continue;
    const size_t pendingToggles = want ? count - ctx->objActiveCount[idx] : ctx->objActiveCount[idx];
    if (pendingToggles == 0) continue;
    if (toggledPrims >= (bypass ? total : general)) continue;
    uint32_t n = 0;
    st = setObject(idx, want, n);
    if (st != NOMAD_OK) return st;
    if (n > 0) toggledPrims = std::min(toggledPrims + n, total);
  }
  bool anyActive = false;
  for (uint32_t o = 0; o < N && !anyActive; ++o) anyActive = ctx->instances[o].primitive_count > 0 && active(o);
  if (!anyActive)
    for (uint32_t idx : order) {
      if (ctx->instances[idx].primitive_count == 0) continue;
      uint32_t n = 0;
      st = setObject(idx, true, n);
      if (st != NOMAD_OK) return st;
      if (n > 0) {
        anyActive = true;
        break;
      }
    }
  if (!anyActive && ctx->primCount > 0) {
    int32_t changed = 0;
    st = nomad_residency_set_primitive_active(ctx, 0, 1, &changed);
    if (st != NOMAD_OK) return st;
  }
  st = nomad_residency_flush(ctx);
  if (st != NOMAD_OK) return st;
  *toggled = (uint32_t)toggledPrims;
  return NOMAD_OK;
}

// updateEnergyImportance (RendererResidency.cpp:1344-2239), its object path for scenes without
// mesh groups (:1462-1860), over the device posterior and ray-hit score of the same step.
// Per object: the summed primitive importance (area times emitted + diffuse + specular +
// transmitted luminance, primitiveImportance Renderer.cpp:1482-1490), raised by the visibility
// boost with the object's screen coverage, times a transport boost from its hit probability,
// normalised ray-hit score, visibility and normalised emitted power, smoothed over steps and
// divided by the primitive count; objects are wanted in that order until min_active primitives
// and the target share of the importance are reached, and toggled in index order under a
// primitive budget and two cooldowns (the per-step object cooldown and the minimum residency
// duration since the last change, :1664-1678). No depth weights are configured (weight 1).
nomad_status energy_step(nomad_ctx *ctx, const nomad_residency_params *prm, const nomad_view &view,
                         uint32_t *toggled) {
  auto &R = ctx->res;
  const uint32_t N = ctx->objectCount;
  if (!toggled) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the EnergyImportance policy runs synchronously");
  if (N > kMaxSelectObjects)
    return nomad_fail(ctx, NOMAD_ERR_LIMIT, "the residency policies support at most 16384 objects");
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (!R.testsOn) {
    R.testsOn = true;
    ctx->frame.clearGraphs();  // the frame now also counts rays tested per object
  }
  if (R.objCooldown.size() != N) R.objCooldown.assign(N, 0);
  if (R.lodDist.size() != N) R.lodDist.assign(N, 0.0f);
  if (R.lodFlags.size() != N) R.lodFlags.assign(N, 0);
  if (R.lastToggle.size() != N) R.lastToggle.assign(N, 0);
  R.lodOn = true;  // nomad_residency_object_state reports this step's coverage and frustum flags
  bool resetHistory = false;
  if (R.energyHist.size() != N) {
    R.energyHist.assign(N, 0.0f);
    resetHistory = true;
  }
  if (R.energyTotal.size() != N) {
    // static per-object sums over the primitives (primitiveImportance and the emitted power times
    // the area), in primitive order, and their total over the scene (_totalPrimitiveImportance)
    R.energyTotal.assign(N, 0.0f);
    R.energyEmit.assign(N, 0.0f);
    std::vector<float> perPrim(ctx->primCount, 0.0f), perEmit(ctx->primCount, 0.0f);
    const float *Pp = ctx->hostPrims.data(), *Mm = ctx->hostMaterials.data();
    auto lum = [](const float *c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; };
    constexpr float kPi = 3.14159265358979323846f;
    for (uint32_t p = 0; p < ctx->primCount; ++p) {
      const float *g = Pp + 28ull * p, *m = Mm + 20ull * p;
      const int type = (int)g[3];
      float area;
      if (type == 0) {
        area = 4.0f * kPi * g[4] * g[4];
      } else {
        float ax, ay, az, bx, by, bz;
        if (type == 1) {
          ax = g[4] - g[0]; ay = g[5] - g[1]; az = g[6] - g[2];
          bx = g[8] - g[0]; by = g[9] - g[1]; bz = g[10] - g[2];
        } else {
          ax = g[4]; ay = g[5]; az = g[6];
          bx = g[8]; by = g[9]; bz = g[10];
        }
        const float cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
        const float len = std::sqrt(cx * cx + cy * cy + cz * cz);
        area = type == 1 ? 0.5f * len : 4.0f * len;
      }
      const float emissive = m[11] * lum(m + 8);
      perPrim[p] = std::max(area, 1e-4f) *
                   (emissive + lum(m) * m[3] + lum(m + 4) * m[3] + (1.0f - m[3]) * lum(m + 12));
      perEmit[p] = std::max(emissive * area, 0.0f);
    }
    for (uint32_t o = 0; o < N; ++o) {
      const nomad_instance_record &ir = ctx->instances[o];
      for (uint32_t p = ir.primitive_base; p < ir.primitive_base + ir.primitive_count; ++p) {
        R.energyTotal[o] += std::max(perPrim[p], 0.0f);
        R.energyEmit[o] += perEmit[p];
      }
    }
    R.energyPrimTotal = 0.0f;
    for (float v : perPrim) R.energyPrimTotal += std::max(v, 0.0f);
  }
  for (uint32_t &c : R.objCooldown)
    if (c > 0) --c;
  cudaStream_t s = ctx->stream;
  nomad_status st = object_pass(ctx, prm, &view);
  if (st != NOMAD_OK) return st;
  const uint32_t frameNo = R.frame + 1;
  ++R.frame;
  std::vector<float> post((size_t)N * kPostWords), score(N);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(post.data(), R.post.p, post.size() * 4, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(score.data(), R.score.p, (size_t)N * 4, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  std::vector<float> cov;
  std::vector<uint8_t> inView;
  object_coverage(ctx, view, cov, inView);
  for (uint32_t o = 0; o < N; ++o) {
    R.lodDist[o] = cov[o];
    R.lodFlags[o] = inView[o];
  }
  auto active = [&](uint32_t o) { return ctx->objActiveCount[o] > 0; };
  const size_t primCount = ctx->primCount;
  const float motion = clamp_unit(prm->camera_motion), pressure = clamp_unit(prm->memory_pressure);
  const float targetFraction = std::min(std::max(prm->target_fraction + 0.08f * motion - 0.12f * pressure, 0.65f), 0.97f);
  const size_t budget = std::max<size_t>(
      1, (size_t)std::llround((double)std::max<uint32_t>(prm->max_toggles, 1) *
                              (1.0 + 0.55 * (double)motion + 0.35 * (double)pressure)));
  float screenArea = (float)view.width * (float)view.height;
  if (screenArea <= 0.0f) screenArea = 1.0f;
  const float boost = std::max(prm->energy_visibility_boost, 1.0f);
  const bool applyBoost = boost > 1.0001f;
  float maxEmit = 0.0f, maxHit = 0.0f, boostedTotal = 0.0f;
  std::vector<float> imp(N);
  for (uint32_t o = 0; o < N; ++o) {
    maxEmit = std::max(maxEmit, R.energyEmit[o]);
    maxHit = std::max(maxHit, std::max(score[o], 0.0f));
    if (applyBoost) {
      const float frac = std::min(std::max(cov[o] / screenArea, 0.0f), 1.0f);
      imp[o] = R.energyTotal[o] * (1.0f + (boost - 1.0f) * frac);
      boostedTotal += std::max(imp[o], 0.0f);
    } else {
      imp[o] = R.energyTotal[o];
    }
  }
  auto normByMax = [](float v, float m) { return !(m > 0.0f) ? 0.0f : std::min(std::max(v / m, 0.0f), 1.0f); };
  for (uint32_t o = 0; o < N; ++o) {
    const float hp = std::min(std::max(post[(size_t)o * kPostWords + 2], 0.0f), 1.0f);
    const float rh = normByMax(std::max(score[o], 0.0f), maxHit);
    const float en = normByMax(R.energyEmit[o], maxEmit);
    const float depthWeight = 1.0f, visibleWeight = inView[o] ? 1.0f : 0.0f;
    const float transport = 1.0f + 0.90f * hp + 0.55f * rh + 0.40f * depthWeight + 0.45f * visibleWeight + 0.90f * en;
    imp[o] *= transport;
  }
  const float historyWeight = std::min(std::max(prm->energy_smoothing, 0.0f), 0.999f);
  const float currentWeight = 1.0f - historyWeight;
  std::vector<float> smoothed(N);
  for (uint32_t o = 0; o < N; ++o) {
    float v = imp[o];
    if (historyWeight > 0.0f) {
      const float prev = resetHistory ? imp[o] : R.energyHist[o];
      v = prev * historyWeight + imp[o] * currentWeight;
    }
    R.energyHist[o] = v;
    smoothed[o] = v;
  }
  if (applyBoost) {
    boostedTotal = 0.0f;
    for (float v : smoothed) boostedTotal += std::max(v, 0.0f);
  }
  const float targetBase = applyBoost ? boostedTotal : R.energyPrimTotal;
  const bool average = prm->energy_use_average != 0;
  std::vector<float> sel(N, 0.0f);
  float totalSel = 0.0f;
  for (uint32_t o = 0; o < N; ++o) {
    const uint32_t count = ctx->instances[o].primitive_count;
    float v = smoothed[o];
    if (average) {
      if (count == 0) continue;
      v /= (float)count;
    }
    sel[o] = v;
    totalSel += std::max(v, 0.0f);
  }
  std::vector<uint32_t> order(N);
  std::iota(order.begin(), order.end(), 0u);
  std::sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) {
    const float sa = sanitize(sel[a]), sb = sanitize(sel[b]);
    if (sa == sb) return a < b;
    return sa > sb;
  });
  const size_t minActive = std::min<size_t>(primCount, prm->min_active);
  std::vector<uint8_t> desired(N, 0);
  size_t enabled = 0;
  if (R.energyPrimTotal <= 0.0f) {
    for (uint32_t idx : order) {
      const uint32_t count = ctx->instances[idx].primitive_count;
      if (count == 0) continue;
      desired[idx] = 1;
      enabled += count;
      if (enabled >= minActive) break;
    }
  } else {
    float cumulative = 0.0f;
    const float target = (totalSel > 0.0f ? totalSel : targetBase) * targetFraction;
    for (uint32_t idx : order) {
      const uint32_t count = ctx->instances[idx].primitive_count;
      if (count == 0 && sel[idx] <= 0.0f) continue;
      desired[idx] = 1;
      enabled += count;
      cumulative += std::max(sel[idx], 0.0f);
      if (enabled >= minActive && cumulative >= target) break;
    }
  }
  if (enabled < minActive)
    for (uint32_t idx : order) {
      if (desired[idx]) continue;
      const uint32_t count = ctx->instances[idx].primitive_count;
      if (count == 0) continue;
      desired[idx] = 1;
      enabled += count;
      if (enabled >= minActive) break;
    }
  size_t toggledPrims = 0;
  const uint32_t minDuration = prm->state_cooldown;
  auto attempt = [&](uint32_t o, bool want, uint32_t &n) -> nomad_status {
    n = 0;
    if (want == active(o)) return NOMAD_OK;
    if (R.objCooldown[o] > 0) return NOMAD_OK;
    if (minDuration > 0 && R.lastToggle[o] != 0 && frameNo >= R.lastToggle[o] && frameNo - R.lastToggle[o] < minDuration)
      return NOMAD_OK;
    const uint32_t count = ctx->instances[o].primitive_count;
    const size_t needed = want ? count - ctx->objActiveCount[o] : ctx->objActiveCount[o];
    if (needed == 0) return NOMAD_OK;
    if (toggledPrims >= budget) return NOMAD_OK;
    const bool prevState = active(o);
    nomad_status r = nomad_residency_set_object_active(ctx, o, want ? 1 : 0, &n);
    if (r != NOMAD_OK) return r;
    const bool newState = active(o);
    if (prevState != newState) R.lastToggle[o] = frameNo;
    if (n > 0 || prevState != newState || !newState) R.objCooldown[o] = prm->state_cooldown;
    if (n > 0) toggledPrims = std::min(toggledPrims + n, budget);
    return NOMAD_OK;
  };
  for (uint32_t o = 0; o < N; ++o) {
    uint32_t n = 0;
    st = attempt(o, desired[o] != 0, n);
    if (st != NOMAD_OK) return st;
  }
  bool anyActive = false;
  for (uint32_t o = 0; o < N && !anyActive; ++o) anyActive = ctx->instances[o].primitive_count > 0 && active(o);
  if (!anyActive)
    for (uint32_t idx : order) {
      if (ctx->instances[idx].primitive_count == 0) continue;
      uint32_t n = 0;
      st = attempt(idx, true, n);
      if (st != NOMAD_OK) return st;
      if (n > 0) {
        anyActive = true;
        break;
      }
    }
  if (!anyActive) {
    uint32_t fb = N;
    for (uint32_t idx : order)
      if (ctx->instances[idx].primitive_count > 0) {
        fb = idx;
        break;
      }
    if (fb < N) {
      uint32_t n = 0;
      st = attempt(fb, true, n);
      if (st != NOMAD_OK) return st;
    } else if (ctx->primCount > 0) {
      int32_t changed = 0;
      st = nomad_residency_set_primitive_active(ctx, 0, 1, &changed);
      if (st != NOMAD_OK) return st;
    }
  }
  st = nomad_residency_flush(ctx);
  if (st != NOMAD_OK) return st;
  *toggled = (uint32_t)toggledPrims;
  return NOMAD_OK;
}

}  // namespace

extern "C" nomad_status nomad_residency_step(nomad_ctx *ctx, const nomad_residency_params *prm,
                                             const nomad_view *camera, uint32_t *toggled) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady || !ctx->res.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (!prm || !camera) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "null parameters or camera");
  if (prm->policy == NOMAD_POLICY_RAYHIT_PRIM) {
    NOMAD_DEVICE_SCOPE(ctx);
    return rayhit_prim_step(ctx, prm, *camera, toggled);
  }
  if (prm->policy == NOMAD_POLICY_DISTANCE_LOD) {
    NOMAD_DEVICE_SCOPE(ctx);
    return distance_lod_step(ctx, prm, *camera, toggled);
  }
  if (prm->policy == NOMAD_POLICY_SCREEN_SPACE) {
    NOMAD_DEVICE_SCOPE(ctx);
    return screen_space_step(ctx, prm, *camera, toggled);
  }
  if (prm->policy == NOMAD_POLICY_PROBABILISTIC) {
    NOMAD_DEVICE_SCOPE(ctx);
    return probabilistic_step(ctx, prm, *camera, toggled);
  }
  if (prm->policy == NOMAD_POLICY_ENERGY) {
    NOMAD_DEVICE_SCOPE(ctx);
    return energy_step(ctx, prm, *camera, toggled);
  }
  if (prm->policy == NOMAD_POLICY_ENVIRONMENT_HIT || prm->policy == NOMAD_POLICY_PREDICTIVE) {
    NOMAD_DEVICE_SCOPE(ctx);
    return environment_step(ctx, prm, *camera, toggled, prm->policy == NOMAD_POLICY_PREDICTIVE);
  }
  if (prm->policy > NOMAD_POLICY_LEARNED) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "unknown policy");
  // Without a usable model the learned policy runs the ray-hit budget step instead.
  nomad_residency_params fallback;
  if (prm->policy == NOMAD_POLICY_LEARNED && !nomad_mlp_ready(ctx)) {
    fallback = *prm;
    fallback.policy = NOMAD_POLICY_RAYHIT_BUDGET;
    prm = &fallback;
    ++ctx->res.fallbackSteps;
  }
  const uint32_t N = ctx->objectCount;
  if (N > kMaxSelectObjects)
    return nomad_fail(ctx, NOMAD_ERR_LIMIT, "device residency selection supports at most 16384 objects");
  NOMAD_DEVICE_SCOPE(ctx);
  auto &R = ctx->res;
  cudaStream_t s = ctx->stream;
  if (!R.testsOn && prm->policy == NOMAD_POLICY_RAYHIT_BUDGET && prm->rayhit_prior_scale > 0.0f) {
    R.testsOn = true;
    ctx->frame.clearGraphs();  // the frame now also counts rays tested per object
  }
  {
    nomad_status ps = object_pass(ctx, prm, camera);
    if (ps != NOMAD_OK) return ps;
  }
  uint32_t npow2 = 1;
  while (npow2 < N) npow2 <<= 1;
  size_t smem = (size_t)npow2 * 10;  // sort keys, selected and candidate flags
  if (smem > 48 * 1024)
    NOMAD_CUDA(ctx, cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  float motion = std::min(std::max(prm->camera_motion, 0.0f), 1.0f);
  uint32_t reserve = (uint32_t)std::min<double>(N, std::ceil(N * (prm->reserve_base + prm->reserve_motion * motion)));
  WidePatch wp{};
  wp.arena = static_cast<int32_t *>(ctx->arena.p);
  for (int w = 0; w < 2; ++w) {
    const nomad::WideLayout &WL = ctx->wide[w];
    // while paging, only the paged layout is on the device
    wp.width[w] = (ctx->pagedWidth && ctx->pagedWidth != WL.width) ? 0u : WL.width;
    wp.fpn[w] = WL.floatsPerNode;
    wp.base[w] = ctx->wideWordBase[w];
    wp.slot[w] = ctx->wideSlot[w].as<const long long>();
    wp.ref[w] = ctx->wideRef[w].as<const int32_t>();
  }
  FrameState &F = ctx->frame;
  LightArgs la{R.emissive.as<const uint4>(), R.emissiveCount, R.primAct.as<const uint8_t>(), F.lightIdx.as<uint32_t>(),
               F.lightCdf.as<float>(), F.lightPdf.as<float>(), F.lightMeta.as<LightMeta>(),
               ctx->prims.as<const float4>(), ctx->materials.as<const float4>(), F.lightRec.as<float4>()};
  // one kernel: selection, toggles, pair and wide layout patches, light CDF
  k_select<<<1, 1024, smem, s>>>(N, npow2, prm->policy, R.keys.as<const float>(), R.visible.as<const uint8_t>(),
                                 R.bytes.as<const unsigned long long>(), prm->budget_bytes, reserve, prm->min_active,
                                 prm->max_toggles, prm->resident_key_bonus, R.desired.as<uint8_t>(),
                                 R.objRes.as<uint8_t>(),
                                 R.objSlot.as<const long long>(), R.objBlasRef.as<const int32_t>(),
                                 static_cast<int32_t *>(ctx->arena.p), R.misc.as<uint32_t>(), wp, la);
  NOMAD_CUDA(ctx, cudaGetLastError());
  F.lightsDirty = false;
  nomad_status st = NOMAD_OK;
  ++R.frame;
  ctx->frame.restirValid = false;
  if (!toggled && ctx->layout.tlasPairCount > 0) {
    // Asynchronous step: the selection kernel patched every layout on the stream; the host mirror
    // is refreshed from a pinned copy when a host call needs it. (Without a TLAS the root ref
    // itself changes and is set on the host: the synchronous path below.)
    if (ctx->resPinnedBytes < N) {
      if (ctx->resPinned) cudaFreeHost(ctx->resPinned);
      ctx->resPinned = nullptr;
      ctx->resPinnedBytes = 0;
      NOMAD_CUDA(ctx, cudaMallocHost(&ctx->resPinned, N));
      ctx->resPinnedBytes = N;
    }
    if (!ctx->resEvent) NOMAD_CUDA(ctx, cudaEventCreateWithFlags(&ctx->resEvent, cudaEventDisableTiming));
    NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->resPinned, R.objRes.p, N, cudaMemcpyDeviceToHost, s));
    NOMAD_CUDA(ctx, cudaEventRecord(ctx->resEvent, s));
    ctx->resHostStale = true;
    return NOMAD_OK;
  }
  // host mirror of the object residency
  uint32_t misc[3];
  NOMAD_CUDA(ctx, cudaMemcpyAsync(misc, R.misc.p, 12, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->objResident.data(), R.objRes.p, N, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  if (misc[1]) {
    for (uint32_t o = 0; o < N; ++o)
      if (ctx->layout.objSlot[o] == -1) ctx->scene.rootRef = misc[2] ? ctx->layout.objBlasRef[o] : kEmptyRef;
  }
  for (uint32_t o = 0; o < N; ++o)
    ctx->instances[o].blas_root_index = ctx->objResident[o] ? ctx->layout.objRootNode[o] : -1;
  st = nomad_patch_wide(ctx);
  if (st != NOMAD_OK) return st;
  ctx->resHostStale = false;
  if (toggled) *toggled = misc[0];
  return NOMAD_OK;
}

nomad_status nomad_residency_sync_host(nomad_ctx *ctx) {
  if (!ctx->resHostStale) return NOMAD_OK;
  NOMAD_CUDA(ctx, cudaEventSynchronize(ctx->resEvent));
  ctx->resHostStale = false;
  const uint32_t N = ctx->objectCount;
  std::memcpy(ctx->objResident.data(), ctx->resPinned, N);
  for (uint32_t o = 0; o < N; ++o)
    ctx->instances[o].blas_root_index = ctx->objResident[o] ? ctx->layout.objRootNode[o] : -1;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_object_bytes(nomad_ctx *ctx, uint64_t *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->res.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  std::memcpy(out, ctx->res.hostBytes.data(), ctx->objectCount * 8ull);
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_last(nomad_ctx *ctx, float *features, float *scores) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->res.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  auto &R = ctx->res;
  if (features)
    NOMAD_CUDA(ctx, cudaMemcpyAsync(features, R.features.p, (size_t)ctx->objectCount * NOMAD_FEATURES * 4,
                                    cudaMemcpyDeviceToHost, ctx->stream));
  if (scores)
    NOMAD_CUDA(ctx, cudaMemcpyAsync(scores, R.keys.p, (size_t)ctx->objectCount * 4, cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_flags(nomad_ctx *ctx, uint8_t *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  nomad_status st = nomad_residency_sync_host(ctx);
  if (st != NOMAD_OK) return st;
  std::memcpy(out, ctx->objResident.data(), ctx->objectCount);
  return NOMAD_OK;
}
