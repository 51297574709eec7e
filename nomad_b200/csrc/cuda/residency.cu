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
// Changes for the B200 build (documented in the design notes): the unit is the object (the
// reference toggles primitives), the target is a geometry byte budget rather than a primitive
// fraction (greedy in score order, skipping objects that do not fit), and the Beta-posterior
// prior is not applied (it needs per-object leaf-test counts whose values depend on traversal
// order).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "rt_context.h"

using namespace nomad_dev;

namespace {

constexpr int kHist = 8;
constexpr uint32_t kMaxSelectObjects = 16384;

struct CamDev {
  float pos[3], fwd[3], right[3], up[3];
  float halfW, halfH, speed;
};

// misc words: [0] toggles, [1] root toggled flag, [2] root resident, [3] total hits this frame,
// [4] total hits previous frame
__global__ void k_features(uint32_t n, CamDev cam, const float4 *__restrict__ bounds,
                           const unsigned long long *__restrict__ bytes, const uint32_t *__restrict__ tris,
                           const float *__restrict__ emit, const uint8_t *__restrict__ res,
                           uint32_t *__restrict__ hits, uint32_t *__restrict__ hist, float *__restrict__ score,
                           uint32_t *__restrict__ lastHit, float *__restrict__ prevDist,
                           uint8_t *__restrict__ visible, float *__restrict__ feat, float *__restrict__ keys,
                           uint32_t *__restrict__ misc, uint32_t frame, float decay, float memPressure) {
  uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  uint32_t h = hits[o];
  hits[o] = 0;
  if (h) atomicAdd(&misc[3], h);
  hist[o * kHist + frame % kHist] = h;
  float s = score[o] * decay + (float)h;
  score[o] = s;
  if (h) lastHit[o] = frame;
  float4 b = bounds[o];
  float dx = b.x - cam.pos[0], dy = b.y - cam.pos[1], dz = b.z - cam.pos[2];
  float dist = sqrtf(dx * dx + dy * dy + dz * dz);
  float z = dx * cam.fwd[0] + dy * cam.fwd[1] + dz * cam.fwd[2];
  float x = dx * cam.right[0] + dy * cam.right[1] + dz * cam.right[2];
  float y = dx * cam.up[0] + dy * cam.up[1] + dz * cam.up[2];
  float r = b.w;
  bool vis = z > -r && fabsf(x) - cam.halfW * z <= r * sqrtf(1.0f + cam.halfW * cam.halfW) &&
             fabsf(y) - cam.halfH * z <= r * sqrtf(1.0f + cam.halfH * cam.halfH);
  visible[o] = vis ? 1 : 0;
  float* f = feat + (size_t)o * NOMAD_FEATURES;
  float zc = fmaxf(z, 1e-3f);
  f[0] = log1pf(dist);
  f[1] = fminf(r / (fmaxf(dist, 1e-3f) * cam.halfH), 4.0f);
  f[2] = vis ? 1.0f : 0.0f;
  for (int k = 0; k < kHist; ++k) f[3 + k] = log1pf((float)hist[o * kHist + (frame + kHist - k) % kHist]);
  f[11] = log1pf(s);
  f[12] = log1pf((float)tris[o]);
  f[13] = log1pf((float)bytes[o] / 1024.0f);
  f[14] = log1pf(emit[o]);
  f[15] = cam.speed;
  f[16] = dist > 0.0f ? z / dist : 1.0f;
  f[17] = log1pf(r);
  f[18] = res[o] ? 1.0f : 0.0f;
  f[19] = log1pf((float)min(frame - lastHit[o], 255u));
  f[20] = (float)h / fmaxf(1.0f, (float)misc[4]);
  f[21] = prevDist[o] > 0.0f ? prevDist[o] - dist : 0.0f;
  f[22] = fminf(fabsf(x) / (zc * cam.halfW), 4.0f);
  f[23] = fminf(fabsf(y) / (zc * cam.halfH), 4.0f);
  prevDist[o] = dist;
  // ray-hit-budget key (RendererResidency.cpp:2833-2840)
  float key = s;
  if (!vis) key = (h == 0) ? 0.0f : key * (0.5f + (0.2f - 0.5f) * memPressure);
  else if (key <= 0.0f) key = 1.0f;
  keys[o] = key;
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

// Greedy fill in sorted order by one warp: candidates (cand[k] = 1) are taken while they fit in
// the budget, skipping those that do not (the sequential rule), 32 positions at a time. Each round
// first drops lanes that cannot fit on their own, then accepts the longest run of candidates whose
// running byte total fits; the first candidate past that run is skipped.
__device__ void warp_greedy(uint32_t n, const unsigned long long *__restrict__ sk,
                            const unsigned long long *__restrict__ bytes, unsigned long long budget, bool unlimited,
                            uint8_t *cand, uint8_t *dsel, unsigned long long *used) {
  const unsigned lane = threadIdx.x & 31u;
  unsigned long long u = *used;
  for (uint32_t base = 0; base < n; base += 32) {
    const uint32_t k = base + lane;
    bool c = k < n && cand[k];
    const unsigned long long b = c ? bytes[(uint32_t)(sk[k] & 0xffffffffu)] : 0ull;
    for (;;) {
      const unsigned long long rem = unlimited ? ~0ull : (u > budget ? 0ull : budget - u);
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
      const bool take = c && (int)lane < f;
      if (take) dsel[k] = 1;
      // bytes taken this round: the prefix just before the first failing lane (or the total)
      const unsigned long long pf = __shfl_sync(0xffffffffu, p, f < 32 ? f : 31);
      const unsigned long long bf = __shfl_sync(0xffffffffu, b, f < 32 ? f : 31);
      u += f < 32 ? pf - bf : pf;
      c = c && (int)lane > f;
    }
  }
  if (lane == 0) *used = u;
}

// Single block of 1024 threads: sort by score, select under the budget (min_active, visibility
// reserve, fill), apply toggles in index order and patch the TLAS refs. Every pass but the two
// budget walks is data-parallel; the budget walks run on one warp, 32 objects at a time.
__global__ void __launch_bounds__(1024) k_select(uint32_t n, uint32_t npow2, uint32_t policy,
                                                 const float *__restrict__ keys, const uint8_t *__restrict__ visible,
                                                 const unsigned long long *__restrict__ bytes,
                                                 unsigned long long budget, uint32_t reserve, uint32_t minActive,
                                                 uint32_t maxToggles, uint8_t *__restrict__ desired,
                                                 uint8_t *__restrict__ res, const long long *__restrict__ slot,
                                                 const int32_t *__restrict__ blasRef, int32_t *__restrict__ pnodeWords,
                                                 uint32_t *__restrict__ misc) {
  extern __shared__ unsigned long long sk[];
  uint8_t *dsel = reinterpret_cast<uint8_t *>(sk + npow2);  // selected, by sorted position
  uint8_t *cand = dsel + npow2;                             // candidates of the current walk
  __shared__ uint32_t warpSums[32];
  __shared__ uint32_t total;
  __shared__ unsigned long long used;
  for (uint32_t i = threadIdx.x; i < npow2; i += blockDim.x)
    sk[i] = i < n ? sort_key(policy == NOMAD_POLICY_ALWAYS ? 1.0f : keys[i], i) : ~0ull;
  if (threadIdx.x == 0) used = 0;
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
  const bool unlimited = budget == 0 || policy == NOMAD_POLICY_ALWAYS;
  // min_active: the best-scored objects stay whatever the budget
  for (uint32_t k = threadIdx.x; k < npow2; k += blockDim.x) {
    const bool m = k < n && k < minActive;
    dsel[k] = m ? 1 : 0;
    if (m) atomicAdd(&used, bytes[(uint32_t)(sk[k] & 0xffffffffu)]);
  }
  __syncthreads();
  // visibility reserve: the first `reserve` visible objects in score order (a contiguous segment
  // of sorted positions per thread, so the scan keeps the sorted order)
  const uint32_t per = (npow2 + blockDim.x - 1) / blockDim.x;
  const uint32_t k0 = threadIdx.x * per;
  uint32_t nv = 0;
  for (uint32_t k = k0; k < k0 + per && k < n; ++k) nv += visible[(uint32_t)(sk[k] & 0xffffffffu)] ? 1u : 0u;
  uint32_t before = block_exscan(nv, warpSums, &total);
  for (uint32_t k = k0; k < k0 + per && k < npow2; ++k) {
    bool c = false;
    if (k < n && visible[(uint32_t)(sk[k] & 0xffffffffu)]) {
      c = before < reserve && !dsel[k];
      ++before;
    }
    cand[k] = c ? 1 : 0;
  }
  __syncthreads();
  if (threadIdx.x < 32) warp_greedy(n, sk, bytes, budget, unlimited, cand, dsel, &used);
  __syncthreads();
  // fill in score order
  for (uint32_t k = threadIdx.x; k < npow2; k += blockDim.x) cand[k] = (k < n && !dsel[k]) ? 1 : 0;
  __syncthreads();
  if (threadIdx.x < 32) warp_greedy(n, sk, bytes, budget, unlimited, cand, dsel, &used);
  __syncthreads();
  for (uint32_t k = threadIdx.x; k < n; k += blockDim.x) desired[(uint32_t)(sk[k] & 0xffffffffu)] = dsel[k];
  __syncthreads();
  // toggles in index order, the first max_toggles of them when bounded
  uint32_t nd = 0;
  for (uint32_t o = k0; o < k0 + per && o < n; ++o) nd += desired[o] != res[o] ? 1u : 0u;
  uint32_t rank = block_exscan(nd, warpSums, &total);
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
  }
  if (threadIdx.x == 0) {
    misc[0] = maxToggles == 0 ? total : min(total, maxToggles);
    misc[4] = misc[3];
    misc[3] = 0;
  }
}

// Light CDF over the emissive primitives whose primitive is active and whose object is
// resident, summed sequentially in primitive order (one thread; the flags are gathered by the
// block first). Also writes the per-primitive light pdf used by ReSTIR.
__global__ void __launch_bounds__(1024) k_lights_rebuild(const uint4 *__restrict__ em, uint32_t ne,
                                                         const uint8_t *__restrict__ primAct,
                                                         const uint8_t *__restrict__ objRes,
                                                         uint32_t *__restrict__ idx, float *__restrict__ cdf,
                                                         float *__restrict__ pdf, LightMeta *__restrict__ meta) {
  __shared__ uint8_t on[4096];
  __shared__ float total_s;
  __shared__ uint32_t count_s;
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
}

float luminance_host(const float *c) { return c[0] * 0.2126f + c[1] * 0.7152f + c[2] * 0.0722f; }

}  // namespace

// Called at scene upload: per-object device arrays, emissive list, bytes, bounds.
nomad_status nomad_residency_init(nomad_ctx *ctx) {
  auto &R = ctx->res;
  const auto &L = ctx->layout;
  const uint32_t N = ctx->objectCount, P = ctx->primCount;
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
    for (size_t i = 0; i < roots.size(); ++i) {
      uint32_t end = i + 1 < roots.size() ? (uint32_t)roots[i + 1].first : R.bvhNodeCount;
      nodes[roots[i].second] = end - (uint32_t)roots[i].first;
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
  NOMAD_CUDA(ctx, F.lightCdf.reserve(std::max<size_t>(1, em.size()) * 4));
  NOMAD_CUDA(ctx, F.lightPdf.reserve((size_t)P * 4));
  NOMAD_CUDA(ctx, F.lightMeta.reserve(sizeof(LightMeta)));
  NOMAD_CUDA(ctx, cudaMemset(F.lightPdf.p, 0, (size_t)P * 4));
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
                                                F.lightMeta.as<LightMeta>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  F.lightsDirty = false;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_step(nomad_ctx *ctx, const nomad_residency_params *prm,
                                             const nomad_view *camera, uint32_t *toggled) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady || !ctx->res.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (!prm || !camera) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "null parameters or camera");
  if (prm->policy > NOMAD_POLICY_LEARNED) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "unknown policy");
  const uint32_t N = ctx->objectCount;
  if (N > kMaxSelectObjects)
    return nomad_fail(ctx, NOMAD_ERR_LIMIT, "device residency selection supports at most 16384 objects");
  NOMAD_CUDA(ctx, cudaSetDevice(ctx->device));
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
  k_features<<<(N + 127) / 128, 128, 0, s>>>(N, cam, R.bounds.as<const float4>(), R.bytes.as<const unsigned long long>(),
                                             R.tris.as<const uint32_t>(), R.emit.as<const float>(),
                                             R.objRes.as<const uint8_t>(), ctx->objHits.as<uint32_t>(),
                                             R.hist.as<uint32_t>(), R.score.as<float>(), R.lastHit.as<uint32_t>(),
                                             R.prevDist.as<float>(), R.visible.as<uint8_t>(), R.features.as<float>(),
                                             R.keys.as<float>(), R.misc.as<uint32_t>(), R.frame, prm->hit_decay,
                                             prm->memory_pressure);
  NOMAD_CUDA(ctx, cudaGetLastError());
  if (prm->policy == NOMAD_POLICY_LEARNED) {
    nomad_status st = nomad_mlp_infer_device(ctx, R.features.as<const float>(), N, R.keys.as<float>());
    if (st != NOMAD_OK) return st;
  }
  uint32_t npow2 = 1;
  while (npow2 < N) npow2 <<= 1;
  size_t smem = (size_t)npow2 * 10;  // sort keys, selected and candidate flags
  NOMAD_CUDA(ctx, cudaFuncSetAttribute(k_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  float motion = std::min(std::max(prm->camera_motion, 0.0f), 1.0f);
  uint32_t reserve = (uint32_t)std::min<double>(N, std::ceil(N * (prm->reserve_base + prm->reserve_motion * motion)));
  NOMAD_CUDA(ctx, cudaMemsetAsync(R.misc.p, 0, 8, s));  // toggles, root flag
  k_select<<<1, 1024, smem, s>>>(N, npow2, prm->policy, R.keys.as<const float>(), R.visible.as<const uint8_t>(),
                                 R.bytes.as<const unsigned long long>(), prm->budget_bytes, reserve, prm->min_active,
                                 prm->max_toggles, R.desired.as<uint8_t>(), R.objRes.as<uint8_t>(),
                                 R.objSlot.as<const long long>(), R.objBlasRef.as<const int32_t>(),
                                 static_cast<int32_t *>(ctx->arena.p), R.misc.as<uint32_t>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  ctx->frame.lightsDirty = true;
  nomad_status st = nomad_lights_update(ctx);
  if (st != NOMAD_OK) return st;
  ++R.frame;
  ctx->frame.restirValid = false;
  if (!toggled && ctx->layout.tlasPairCount > 0) {
    // Asynchronous step: the wide layouts follow the device flags on the stream, the host mirror
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
    st = nomad_patch_wide(ctx);
    if (st != NOMAD_OK) return st;
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
