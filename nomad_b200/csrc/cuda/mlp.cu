// Learned residency scorer: MLP 24 -> 128 -> 128 -> 1 (ReLU), BF16 weights and activations,
// FP32 accumulation on the tensor cores, trained on the device with AdamW. Every matrix product
// runs on tcgen05 with tensor-memory accumulators: inference (every residency step) and the
// training forward pass in one fused kernel (both hidden layers and the output dot product, the
// weights staged by one bulk copy), and the backward products in a tiled GEMM kernel whose
// operands the threads stage in the canonical shared-memory layout.
//
// The GEMMs are tiny (2,048 objects x 128 x 128 per frame; a 4,096-row training batch), so the
// kernels are built for latency; the backward products use split-K partial sums reduced in a
// fixed order, so training is bit-reproducible for a given seed.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <numeric>
#include <random>
#include <vector>

#include "residency_features.cuh"
#include "rt_context.h"

namespace {

constexpr int kIn = NOMAD_FEATURES;  // 24
constexpr int kInPad = 32;
constexpr int kHid = 128;
// offsets in the fp32 parameter blob
constexpr int oW1 = 0;
constexpr int oB1 = oW1 + kHid * kInPad;
constexpr int oW2 = oB1 + kHid;
constexpr int oB2 = oW2 + kHid * kHid;
constexpr int oW3 = oB2 + kHid;
constexpr int oB3 = oW3 + kHid;
constexpr int oMean = oB3 + 1;
constexpr int oIstd = oMean + kIn;
constexpr int kParams = oIstd + kIn;
static_assert(kParams == NOMAD_MLP_PARAMS, "parameter blob layout");

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);  // a -> low half
  return *reinterpret_cast<uint32_t *>(&h);
}

// ---- inference on the 5th-generation tensor cores (tcgen05) ---------------------------------
// One CTA of 128 threads scores 128 rows. Both layers run as tcgen05.mma (kind::f16, BF16 inputs,
// FP32 accumulators in tensor memory, M = 128, N = 128, K = 16 per instruction) issued by one
// thread, with the operands in shared memory in the canonical K-major layout without swizzle:
// 8 x 8 core matrices of 128 contiguous bytes, row groups 128 B apart (stride byte offset) and
// 8-element K chunks (rows / 8) * 128 B apart (leading byte offset). Each thread then owns one
// accumulator row (its tensor-memory lane) for the bias / ReLU epilogue and the final dot product.
constexpr int kTcRows = 128;
constexpr uint32_t kTcCols = 256;                   // tensor-memory columns: D1 [0,128), D2 [128,256)
constexpr uint32_t kTcX = 0;                        // X tile, 128 x 32 bf16
constexpr uint32_t kTcW1 = kTcX + 128 * kInPad * 2; // W1, 128 x 32, then W2 right after it:
constexpr uint32_t kTcW2 = kTcW1 + 128 * kInPad * 2; // both arrive pre-packed in one bulk copy
constexpr uint32_t kTcWBytes = 128 * kInPad * 2 + 128 * kHid * 2;  // 40 KB
constexpr uint32_t kTcH1 = kTcW2 + 128 * kHid * 2;
constexpr uint32_t kTcF = kTcH1 + 128 * kHid * 2;   // fp32: b1, b2, w3, b3, mean, istd
constexpr uint32_t kTcBar = kTcF + 4 * (3 * kHid + 1 + 2 * kIn + 7);  // copy barrier, MMA barrier, TMEM slot
constexpr size_t kTcSmem = kTcBar + 24;
constexpr uint32_t kStatusWaitExpired = 1u << 1;
constexpr long long kTcWaitPolls = 1ll << 22;

// Byte offset of element (r, k) of a 128-row K-major operand in the canonical layout.
__device__ __forceinline__ uint32_t canon_off(int r, int k) {
  return (uint32_t)((((k >> 3) * 16 + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Shared-memory matrix descriptor: start, leading byte offset (next K chunk: 16 row groups of
// 128 B), stride byte offset (next row group: 128 B), descriptor version 1, no swizzle.
__device__ __forceinline__ uint64_t canon_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)(2048u >> 4) << 16) | ((uint64_t)(128u >> 4) << 32) |
         (1ull << 46);
}

// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, N = 128, M = 128.
constexpr uint32_t kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((128u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity) {
  for (long long i = 0; i < kTcWaitPolls; ++i) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// 32 consecutive accumulator columns of this thread's lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}

// Wc holds W1 and W2 (bf16) already in the canonical shared-memory layout (k_refresh_bf16 packs
// them whenever the weights change), so one bulk asynchronous copy stages both.
// FEAT: the rows are the residency step's objects; each thread computes its object's features
// (nomad_res::object_features, the same code as the feature kernel) instead of reading X.
// SAVE (training): also stores what the backward pass needs, row-major: the standardised inputs
// (bf16, n x 32), Z1 = X W1^T + b1 (fp32), H1 = ReLU(Z1) (bf16) and Z2 = H1 W2^T + b2 (fp32).
struct FwdSave {
  __nv_bfloat16 *xbf, *h1;
  float *z1, *z2;
};

template <bool FEAT, bool SAVE>
__global__ void __launch_bounds__(128) k_mlp_forward_tc(const float *__restrict__ X, uint64_t n,
                                                        const float *__restrict__ P,
                                                        const unsigned char *__restrict__ Wc, float *__restrict__ y,
                                                        uint32_t *__restrict__ status, nomad_res::FeatArgs fa,
                                                        FwdSave sv) {
  extern __shared__ __align__(16) unsigned char smem[];
  const uint32_t sbase = static_cast<uint32_t>(__cvta_generic_to_shared(smem));
  float *sB1 = reinterpret_cast<float *>(smem + kTcF);
  float *sB2 = sB1 + kHid;
  float *sW3 = sB2 + kHid;
  float *sB3 = sW3 + kHid;
  float *sMean = sB3 + 1;
  float *sIstd = sMean + kIn;
  const uint32_t barCopy = sbase + kTcBar, bar = sbase + kTcBar + 8;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + kTcBar + 16);
  const int tid = threadIdx.x, warp = tid >> 5;

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(barCopy) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    // weights: one bulk copy (no multicast) of the pre-packed W1 | W2 block
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(barCopy), "r"(kTcWBytes) : "memory");
    for (uint32_t off = 0; off < kTcWBytes; off += 16384u) {
      const uint32_t sz = min(16384u, kTcWBytes - off);
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              sbase + kTcW1 + off),
          "l"(Wc + off), "r"(sz), "r"(barCopy)
          : "memory");
    }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kTcBar + 16),
                 "r"(kTcCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // the standardised X tile and the fp32 vectors while the weights are in flight
  for (int i = tid; i < kHid; i += 128) {
    sB1[i] = P[oB1 + i];
    sB2[i] = P[oB2 + i];
    sW3[i] = P[oW3 + i];
  }
  if (tid == 0) sB3[0] = P[oB3];
  if (tid < kIn) {
    sMean[tid] = P[oMean + tid];
    sIstd[tid] = P[oIstd + tid];
  }
  __syncthreads();
  const uint64_t row0 = (uint64_t)blockIdx.x * kTcRows;
  if constexpr (FEAT) {
    float f[NOMAD_FEATURES];
    const bool live = row0 + tid < n;
    if (live) nomad_res::object_features(fa, (uint32_t)(row0 + tid), f);
#pragma unroll
    for (int k = 0; k < kInPad; ++k) {
      const float v = (live && k < kIn) ? (f[k < kIn ? k : 0] - sMean[k < kIn ? k : 0]) * sIstd[k < kIn ? k : 0] : 0.0f;
      *reinterpret_cast<__nv_bfloat16 *>(smem + kTcX + canon_off(tid, k)) = __float2bfloat16_rn(v);
    }
  } else {
    for (int i = tid; i < kTcRows * kInPad; i += 128) {
      const int r = i / kInPad, f = i % kInPad;
      float v = 0.0f;
      if (f < kIn && row0 + r < n) v = (X[(row0 + r) * kIn + f] - sMean[f]) * sIstd[f];
      const __nv_bfloat16 b = __float2bfloat16_rn(v);
      *reinterpret_cast<__nv_bfloat16 *>(smem + kTcX + canon_off(r, f)) = b;
      if (SAVE && row0 + r < n) sv.xbf[(row0 + r) * kInPad + f] = b;
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
  bool ok = tc_wait(barCopy, 0);  // weights landed

  // layer 1: D1 = X . W1^T, K = 32 in two steps
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < kInPad / 16; ++s)
      tc_mma(tmem, canon_desc(sbase + kTcX + s * 2 * 2048), canon_desc(sbase + kTcW1 + s * 2 * 2048), s > 0);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
  }
  ok = tc_wait(bar, 0) && ok;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // epilogue 1: bias, ReLU, BF16 into the layer-2 operand (row = this thread's lane)
  const int r = tid;
  const bool rowLive = row0 + r < n;
#pragma unroll
  for (int c0 = 0; c0 < kHid; c0 += 32) {
    float v[32];
    tc_ld32(lane_base + c0, v);
#pragma unroll
    for (int j = 0; j < 32; j += 2) {
      const float za = v[j] + sB1[c0 + j], zb = v[j + 1] + sB1[c0 + j + 1];
      const uint32_t h = pack_bf16(fmaxf(za, 0.0f), fmaxf(zb, 0.0f));
      *reinterpret_cast<uint32_t *>(smem + kTcH1 + canon_off(r, c0 + j)) = h;
      if (SAVE && rowLive) {
        const uint64_t o = (row0 + r) * kHid + c0 + j;
        sv.z1[o] = za;
        sv.z1[o + 1] = zb;
        *reinterpret_cast<uint32_t *>(sv.h1 + o) = h;
      }
    }
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // layer 2: D2 = H1 . W2^T, K = 128 in eight steps
  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < kHid / 16; ++s)
      tc_mma(tmem + 128, canon_desc(sbase + kTcH1 + s * 2 * 2048), canon_desc(sbase + kTcW2 + s * 2 * 2048), s > 0);
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
  }
  ok = tc_wait(bar, 1) && ok;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  // epilogue 2: ReLU(D2 + b2) . w3 + b3 for this thread's row
  float acc = 0.0f;
#pragma unroll
  for (int c0 = 0; c0 < kHid; c0 += 32) {
    float v[32];
    tc_ld32(lane_base + 128 + c0, v);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      const float z = v[j] + sB2[c0 + j];
      if (SAVE && rowLive) sv.z2[(row0 + r) * kHid + c0 + j] = z;
      acc += fmaxf(z, 0.0f) * sW3[c0 + j];
    }
  }
  if (row0 + r < n) y[row0 + r] = ok ? acc + sB3[0] : 0.0f;
  if (!ok && tid == 0) atomicOr(status, kStatusWaitExpired);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTcCols) : "memory");
  }
}

// ---- backward GEMMs on the 5th-generation tensor cores (tcgen05) ---------------------------
// C[z][M][N] (fp32) = sum over split z's K range of op(A)[M][K] op(B)[K][N], where A is stored
// [M][K] (TA = 0) or [K][M] (TA = 1) and B [K][N] (TB = 0) or [N][K] (TB = 1), all bf16. One CTA
// of 128 threads owns a 128-row tile of C and all NT (= N rounded up: 32 or 128) columns,
// accumulated in tensor memory. K advances 64 at a time: the threads stage the A tile (128 x 64)
// and the B tile (NT x 64) in shared memory in the canonical K-major layout (whatever the global
// layout, so transposed operands cost nothing extra), then one thread issues four
// tcgen05.mma (M = 128, N = NT, K = 16) and commits to an mbarrier that every thread waits on
// before the tiles are overwritten. Elements past M, N or the split's K range are staged as zero.
// Split-K partial tiles are summed afterwards in a fixed order (k_reduce_splits), so a gradient
// is bit-reproducible.
constexpr int kGemmK = 64;

// Byte offset of element (r, k) of an R-row K-major operand tile in the canonical layout.
template <int R>
__device__ __forceinline__ uint32_t canon_off_r(int r, int k) {
  return (uint32_t)((((k >> 3) * (R / 8) + (r >> 3)) << 7) + ((r & 7) << 4) + ((k & 7) << 1));
}

// Descriptor of an R-row operand: next K chunk (R / 8) * 128 B away, next row group 128 B away.
template <int R>
__device__ __forceinline__ uint64_t canon_desc_r(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3fffu) | ((uint64_t)((R / 8 * 128) >> 4) << 16) |
         ((uint64_t)(128u >> 4) << 32) | (1ull << 46);
}

template <int NT>
__device__ __forceinline__ void tc_mma_n(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  // kind::f16: FP32 accumulator, BF16 A and B, both K-major, N = NT, M = 128
  constexpr uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) | ((128u >> 4) << 24);
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

template <bool TA, bool TB, int NT>
__global__ void __launch_bounds__(128) k_gemm_tc(const __nv_bfloat16 *__restrict__ A,
                                                 const __nv_bfloat16 *__restrict__ B, float *__restrict__ C,
                                                 int M, int N, int K, int lda, int ldb, int kPerSplit,
                                                 uint32_t *__restrict__ status) {
  static_assert(NT == 32 || NT == 64 || NT == 128, "tile width");
  __shared__ __align__(1024) unsigned char sA[128 * kGemmK * 2];
  __shared__ __align__(1024) unsigned char sB[NT * kGemmK * 2];
  __shared__ __align__(8) unsigned long long sBar;
  __shared__ uint32_t sTmem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t aBase = static_cast<uint32_t>(__cvta_generic_to_shared(sA));
  const uint32_t bBase = static_cast<uint32_t>(__cvta_generic_to_shared(sB));
  const uint32_t bar = static_cast<uint32_t>(__cvta_generic_to_shared(&sBar));
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     static_cast<uint32_t>(__cvta_generic_to_shared(&sTmem))),
                 "r"((uint32_t)NT)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = sTmem;
  const int m0 = blockIdx.y * 128;
  const int kBeg = blockIdx.z * kPerSplit, kEnd = min(K, kBeg + kPerSplit);
  const __nv_bfloat16 zero = __float2bfloat16_rn(0.0f);
  uint32_t phase = 0;
  bool ok = true, issued = false;
  for (int k0 = kBeg; k0 < kEnd && ok; k0 += kGemmK) {
    for (int i = tid; i < 128 * kGemmK; i += 128) {
      // consecutive threads read consecutive addresses of the stored layout
      const int r = TA ? i % 128 : i / kGemmK, c = TA ? i / 128 : i % kGemmK;
      const int m = m0 + r, k = k0 + c;
      __nv_bfloat16 v = zero;
      if (m < M && k < kEnd) v = TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
      *reinterpret_cast<__nv_bfloat16 *>(sA + canon_off_r<128>(r, c)) = v;
    }
    for (int i = tid; i < NT * kGemmK; i += 128) {
      const int r = TB ? i / kGemmK : i % NT, c = TB ? i % kGemmK : i / NT;
      const int k = k0 + c;
      __nv_bfloat16 v = zero;
      if (r < N && k < kEnd) v = TB ? B[(size_t)r * ldb + k] : B[(size_t)k * ldb + r];
      *reinterpret_cast<__nv_bfloat16 *>(sB + canon_off_r<NT>(r, c)) = v;
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
#pragma unroll
      for (int s = 0; s < kGemmK / 16; ++s)
        tc_mma_n<NT>(tmem, canon_desc_r<128>(aBase + s * 2 * (128 / 8 * 128)),
                     canon_desc_r<NT>(bBase + s * 2 * (NT / 8 * 128)), (k0 > kBeg || s > 0) ? 1u : 0u);
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                   : "memory");
    }
    issued = true;
    ok = __syncthreads_and(tc_wait(bar, phase) ? 1 : 0) != 0;  // one outcome for the whole CTA
    phase ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  if (!ok) {
    // the last commit did not arrive in time: give the MMAs in flight one more bounded wait
    // before the tensor memory is released, and report it
    tc_wait(bar, phase ^ 1u);
    if (tid == 0) atomicOr(status, kStatusWaitExpired);
  }
  const int row = m0 + tid;
  float *Cz = C + (size_t)blockIdx.z * M * N;
  const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
  for (int c0 = 0; c0 < NT; c0 += 32) {
    float v[32];
    if (issued) {
      tc_ld32(lane_base + c0, v);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = 0.0f;  // empty K range
    }
    if (row < M) {
#pragma unroll
      for (int j = 0; j < 32; ++j)
        if (c0 + j < N) Cz[(size_t)row * N + c0 + j] = ok ? v[j] : 0.0f;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)NT) : "memory");
  }
}

// Sums split-K partials in fixed order: out[i] = sum_z part[z][i].
__global__ void k_reduce_splits(const float *__restrict__ part, int splits, size_t count,
                                float *__restrict__ out) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
    float s = 0.0f;
    for (int z = 0; z < splits; ++z) s += part[(size_t)z * count + i];
    out[i] = s;
  }
}

// dy = 2 (y - t) / B; per-row squared errors for the loss.
__global__ void k_mse_grad(const float *__restrict__ y, const float *__restrict__ t, int B,
                           float *__restrict__ dy, float *__restrict__ se) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B) {
    float d = y[i] - t[i];
    dy[i] = 2.0f * d / (float)B;
    se[i] = d * d;
  }
}

// dZ2 = dy * w3 * (Z2 > 0) (bf16 for the GEMMs, fp32 kept for the bias gradient).
__global__ void k_dz2(const float *__restrict__ dy, const float *__restrict__ z2, const float *__restrict__ P,
                      int B, __nv_bfloat16 *__restrict__ dz2b, float *__restrict__ dz2f) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B * kHid) {
    int r = i / kHid, c = i % kHid;
    float v = z2[i] > 0.0f ? dy[r] * P[oW3 + c] : 0.0f;
    dz2f[i] = v;
    dz2b[i] = __float2bfloat16_rn(v);
  }
}

// dZ1 = dH1 * (Z1 > 0).
__global__ void k_dz1(const float *__restrict__ dh1, const float *__restrict__ z1, int B,
                      __nv_bfloat16 *__restrict__ dz1b, float *__restrict__ dz1f) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B * kHid) {
    float v = z1[i] > 0.0f ? dh1[i] : 0.0f;
    dz1f[i] = v;
    dz1b[i] = __float2bfloat16_rn(v);
  }
}

// Column sums in fixed row order: out[c] = sum_r M[r][c] * (w ? w[r] : 1); one thread per column.
__global__ void k_colsum(const float *__restrict__ M, const float *__restrict__ w, int rows, int cols,
                         float *__restrict__ out) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < cols) {
    float s = 0.0f;
    for (int r = 0; r < rows; ++r) s += M[(size_t)r * cols + c] * (w ? w[r] : 1.0f);
    out[c] = s;
  }
}

// AdamW over the trainable part of the blob (everything before the feature statistics).
__global__ void k_adamw(float *__restrict__ P, const float *__restrict__ G, float *__restrict__ m,
                        float *__restrict__ v, int count, float lr, float b1, float b2, float eps,
                        float wd, float bc1, float bc2) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) {
    float g = G[i];
    float mi = b1 * m[i] + (1.0f - b1) * g;
    float vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    float mh = mi / bc1, vh = vi / bc2;
    bool isWeight = (i < oB1) || (i >= oW2 && i < oB2) || (i >= oW3 && i < oB3);
    float p = P[i];
    if (isWeight) p = p - lr * wd * p;
    P[i] = p - lr * mh / (sqrtf(vh) + eps);
  }
}

// bf16 copies of W1 and W2 (W1's padded input columns stay zero), row-major for the training
// kernels and packed in the canonical layout of the tcgen05 inference kernel (W1 then W2).
__global__ void k_refresh_bf16(const float *__restrict__ P, __nv_bfloat16 *__restrict__ W1b,
                               __nv_bfloat16 *__restrict__ W2b, unsigned char *__restrict__ Wc) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < kHid * kInPad) {
    const __nv_bfloat16 w = __float2bfloat16_rn((i % kInPad) < kIn ? P[oW1 + i] : 0.0f);
    W1b[i] = w;
    *reinterpret_cast<__nv_bfloat16 *>(Wc + canon_off(i / kInPad, i % kInPad)) = w;
  }
  if (i < kHid * kHid) {
    const __nv_bfloat16 w = __float2bfloat16_rn(P[oW2 + i]);
    W2b[i] = w;
    *reinterpret_cast<__nv_bfloat16 *>(Wc + (kTcW2 - kTcW1) + canon_off(i / kHid, i % kHid)) = w;
  }
}

// Gathers a mini-batch of raw features and targets.
__global__ void k_gather(const float *__restrict__ X, const float *__restrict__ T, const uint32_t *__restrict__ idx,
                         int B, float *__restrict__ xb, float *__restrict__ tb) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < B * kIn) xb[i] = X[(size_t)idx[i / kIn] * kIn + i % kIn];
  if (i < B) tb[i] = T[idx[i]];
}

}  // namespace

// ---- host side ------------------------------------------------------------------------------

struct MlpState {
  bool ready = false;
  DeviceBuf P, W1b, W2b, Wc, M, V, G;
  DeviceBuf X, T, idx, xb, tb, y, z1, h1, z2, xbf, dy, se, dz2b, dz2f, dh1, dz1b, dz1f, part;
  uint64_t trainCap = 0;
  int batchCap = 0;
  DeviceBuf inX, inY;
};

namespace {
MlpState &mlp(nomad_ctx *ctx) {
  static_assert(sizeof(MlpState) > 0, "");
  if (!ctx->mlp) ctx->mlp = new MlpState();
  return *static_cast<MlpState *>(ctx->mlp);
}

nomad_status refresh(nomad_ctx *ctx, MlpState &S) {
  int n = kHid * kHid;
  k_refresh_bf16<<<(n + 255) / 256, 256, 0, ctx->stream>>>(S.P.as<const float>(), S.W1b.as<__nv_bfloat16>(),
                                                            S.W2b.as<__nv_bfloat16>(), S.Wc.as<unsigned char>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

nomad_status ensure(nomad_ctx *ctx, MlpState &S) {
  NOMAD_CUDA(ctx, S.P.reserve(kParams * 4));
  NOMAD_CUDA(ctx, S.W1b.reserve(kHid * kInPad * 2));
  NOMAD_CUDA(ctx, S.W2b.reserve(kHid * kHid * 2));
  NOMAD_CUDA(ctx, S.Wc.reserve(kTcWBytes));
  NOMAD_CUDA(ctx, S.M.reserve(kParams * 4));
  NOMAD_CUDA(ctx, S.V.reserve(kParams * 4));
  NOMAD_CUDA(ctx, S.G.reserve(kParams * 4));
  static bool attr = false;
  if (!attr) {
    NOMAD_CUDA(ctx, cudaFuncSetAttribute(k_mlp_forward_tc<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmem));
    NOMAD_CUDA(ctx, cudaFuncSetAttribute(k_mlp_forward_tc<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmem));
    NOMAD_CUDA(ctx, cudaFuncSetAttribute(k_mlp_forward_tc<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kTcSmem));
    attr = true;
  }
  return NOMAD_OK;
}
}  // namespace

void nomad_mlp_free(void *p) { delete static_cast<MlpState *>(p); }

// Inference on device features (n x 24 fp32) into y (n fp32), on the context stream.
nomad_status nomad_mlp_infer_device(nomad_ctx *ctx, const float *X, uint64_t n, float *y) {
  MlpState &S = mlp(ctx);
  if (!S.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "MLP not initialised or trained");
  if (n == 0) return NOMAD_OK;
  const unsigned blocks = (unsigned)((n + kTcRows - 1) / kTcRows);
  k_mlp_forward_tc<false, false><<<blocks, 128, kTcSmem, ctx->stream>>>(X, n, S.P.as<const float>(),
                                                                        S.Wc.as<const unsigned char>(), y,
                                                                        ctx->status.as<uint32_t>(),
                                                                        nomad_res::FeatArgs{}, FwdSave{});
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

nomad_status nomad_mlp_score_objects(nomad_ctx *ctx, const nomad_res::FeatArgs *fa, float *keys) {
  MlpState &S = mlp(ctx);
  if (!S.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "MLP not initialised or trained");
  if (fa->n == 0) return NOMAD_OK;
  const unsigned blocks = (fa->n + kTcRows - 1) / kTcRows;
  k_mlp_forward_tc<true, false><<<blocks, 128, kTcSmem, ctx->stream>>>(nullptr, fa->n, S.P.as<const float>(),
                                                                       S.Wc.as<const unsigned char>(), keys,
                                                                       ctx->status.as<uint32_t>(), *fa, FwdSave{});
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

extern "C" nomad_status nomad_mlp_init(nomad_ctx *ctx, uint64_t seed) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  MlpState &S = mlp(ctx);
  nomad_status st = ensure(ctx, S);
  if (st != NOMAD_OK) return st;
  std::vector<float> p(kParams, 0.0f);
  std::mt19937_64 rng(seed);
  auto uni = [&](float lim) { return (float)(((rng() >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0) * lim; };
  float l1 = std::sqrt(6.0f / kIn), l2 = std::sqrt(6.0f / kHid), l3 = std::sqrt(3.0f / kHid);
  for (int o = 0; o < kHid; ++o)
    for (int i = 0; i < kIn; ++i) p[oW1 + o * kInPad + i] = uni(l1);
  for (int i = 0; i < kHid * kHid; ++i) p[oW2 + i] = uni(l2);
  for (int i = 0; i < kHid; ++i) p[oW3 + i] = uni(l3);
  for (int i = 0; i < kIn; ++i) p[oIstd + i] = 1.0f;
  NOMAD_CUDA(ctx, cudaMemcpy(S.P.p, p.data(), kParams * 4, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemset(S.M.p, 0, kParams * 4));
  NOMAD_CUDA(ctx, cudaMemset(S.V.p, 0, kParams * 4));
  st = refresh(ctx, S);
  if (st != NOMAD_OK) return st;
  S.ready = true;
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_mlp_get(nomad_ctx *ctx, float *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  MlpState &S = mlp(ctx);
  if (!S.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "MLP not initialised");
  NOMAD_CUDA(ctx, cudaMemcpyAsync(out, S.P.p, kParams * 4, cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

bool nomad_mlp_ready(nomad_ctx *ctx) { return ctx->mlp && static_cast<MlpState *>(ctx->mlp)->ready; }

extern "C" nomad_status nomad_mlp_set(nomad_ctx *ctx, const float *in) {
  if (!ctx || !in) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  MlpState &S = mlp(ctx);
  for (int i = 0; i < kParams; ++i)
    if (!std::isfinite(in[i])) {
      S.ready = false;
      return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT,
                        "model parameter " + std::to_string(i) +
                            " is not finite; learned steps fall back to the ray-hit budget");
    }
  nomad_status st = ensure(ctx, S);
  if (st != NOMAD_OK) return st;
  NOMAD_CUDA(ctx, cudaMemcpy(S.P.p, in, kParams * 4, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemset(S.M.p, 0, kParams * 4));
  NOMAD_CUDA(ctx, cudaMemset(S.V.p, 0, kParams * 4));
  st = refresh(ctx, S);
  if (st != NOMAD_OK) return st;
  S.ready = true;
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

namespace {
constexpr uint32_t kModelVersion = 1;
constexpr size_t kModelHeader = 16;  // magic, version, parameter count, feature count

uint64_t fnv1a(const unsigned char *p, size_t n) {
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ull;
  }
  return h;
}

void put_u32(unsigned char *p, uint32_t v) {
  for (int k = 0; k < 4; ++k) p[k] = static_cast<unsigned char>(v >> (8 * k));
}

uint32_t get_u32(const unsigned char *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
}  // namespace

extern "C" nomad_status nomad_mlp_save(nomad_ctx *ctx, const char *path) {
  if (!ctx || !path) return NOMAD_ERR_INVALID_ARGUMENT;
  std::vector<float> p(kParams);
  nomad_status st = nomad_mlp_get(ctx, p.data());
  if (st != NOMAD_OK) return st;
  std::vector<unsigned char> buf(kModelHeader + (size_t)kParams * 4 + 8);
  std::memcpy(buf.data(), "NMLP", 4);
  put_u32(buf.data() + 4, kModelVersion);
  put_u32(buf.data() + 8, (uint32_t)kParams);
  put_u32(buf.data() + 12, (uint32_t)kIn);
  for (int i = 0; i < kParams; ++i) {
    uint32_t bits;
    std::memcpy(&bits, &p[i], 4);
    put_u32(buf.data() + kModelHeader + 4 * (size_t)i, bits);
  }
  const size_t body = kModelHeader + (size_t)kParams * 4;
  const uint64_t h = fnv1a(buf.data(), body);
  put_u32(buf.data() + body, (uint32_t)h);
  put_u32(buf.data() + body + 4, (uint32_t)(h >> 32));
  FILE *f = std::fopen(path, "wb");
  if (!f) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  const bool ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed) return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, std::string("cannot write ") + path);
  return NOMAD_OK;
}

extern "C" nomad_status nomad_mlp_load(nomad_ctx *ctx, const char *path) {
  if (!ctx || !path) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  MlpState &S = mlp(ctx);
  auto reject = [&](const std::string &why) {
    S.ready = false;
    return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT,
                      std::string("model file ") + path + ": " + why +
                          "; learned steps fall back to the ray-hit budget");
  };
  const size_t body = kModelHeader + (size_t)kParams * 4;
  std::vector<unsigned char> buf;
  {
    FILE *f = std::fopen(path, "rb");
    if (!f) return reject("cannot be opened");
    unsigned char tmp[65536];
    size_t got;
    while ((got = std::fread(tmp, 1, sizeof(tmp), f)) > 0 && buf.size() <= body + 8)
      buf.insert(buf.end(), tmp, tmp + got);
    std::fclose(f);
  }
  if (buf.size() < kModelHeader || std::memcmp(buf.data(), "NMLP", 4) != 0) return reject("not a model file");
  if (get_u32(buf.data() + 4) != kModelVersion)
    return reject("format version " + std::to_string(get_u32(buf.data() + 4)) + ", expected " +
                  std::to_string(kModelVersion));
  if (get_u32(buf.data() + 8) != (uint32_t)kParams || get_u32(buf.data() + 12) != (uint32_t)kIn)
    return reject("shape differs from this library's model");
  if (buf.size() != body + 8) return reject("size " + std::to_string(buf.size()) + " bytes, expected " +
                                            std::to_string(body + 8));
  const uint64_t want = (uint64_t)get_u32(buf.data() + body) | ((uint64_t)get_u32(buf.data() + body + 4) << 32);
  if (fnv1a(buf.data(), body) != want) return reject("checksum mismatch");
  std::vector<float> p(kParams);
  for (int i = 0; i < kParams; ++i) {
    const uint32_t bits = get_u32(buf.data() + kModelHeader + 4 * (size_t)i);
    std::memcpy(&p[i], &bits, 4);
    if (!std::isfinite(p[i])) return reject("parameter " + std::to_string(i) + " is not finite");
  }
  return nomad_mlp_set(ctx, p.data());
}

extern "C" nomad_status nomad_mlp_infer(nomad_ctx *ctx, const float *features, uint64_t n, float *out,
                                        uint32_t flags) {
  if (!ctx || (!features && n) || (!out && n)) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  MlpState &S = mlp(ctx);
  if (flags & NOMAD_TRACE_DEVICE_POINTERS) return nomad_mlp_infer_device(ctx, features, n, out);
  NOMAD_CUDA(ctx, S.inX.reserve(std::max<uint64_t>(1, n) * kIn * 4));
  NOMAD_CUDA(ctx, S.inY.reserve(std::max<uint64_t>(1, n) * 4));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(S.inX.p, features, n * kIn * 4, cudaMemcpyHostToDevice, ctx->stream));
  nomad_status st = nomad_mlp_infer_device(ctx, S.inX.as<const float>(), n, S.inY.as<float>());
  if (st != NOMAD_OK) return st;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(out, S.inY.p, n * 4, cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

namespace {

nomad_status ensure_batch(nomad_ctx *ctx, MlpState &S, int B, int splits) {
  if (S.batchCap < B) {
    NOMAD_CUDA(ctx, S.idx.reserve((size_t)B * 4));
    NOMAD_CUDA(ctx, S.xb.reserve((size_t)B * kIn * 4));
    NOMAD_CUDA(ctx, S.tb.reserve((size_t)B * 4));
    NOMAD_CUDA(ctx, S.y.reserve((size_t)B * 4));
    NOMAD_CUDA(ctx, S.z1.reserve((size_t)B * kHid * 4));
    NOMAD_CUDA(ctx, S.h1.reserve((size_t)B * kHid * 2));
    NOMAD_CUDA(ctx, S.z2.reserve((size_t)B * kHid * 4));
    NOMAD_CUDA(ctx, S.xbf.reserve((size_t)B * kInPad * 2));
    NOMAD_CUDA(ctx, S.dy.reserve((size_t)B * 4));
    NOMAD_CUDA(ctx, S.se.reserve((size_t)B * 4));
    NOMAD_CUDA(ctx, S.dz2b.reserve((size_t)B * kHid * 2));
    NOMAD_CUDA(ctx, S.dz2f.reserve((size_t)B * kHid * 4));
    NOMAD_CUDA(ctx, S.dh1.reserve((size_t)B * kHid * 4));
    NOMAD_CUDA(ctx, S.dz1b.reserve((size_t)B * kHid * 2));
    NOMAD_CUDA(ctx, S.dz1f.reserve((size_t)B * kHid * 4));
    S.batchCap = B;
  }
  NOMAD_CUDA(ctx, S.part.reserve((size_t)std::max(splits, 1) * kHid * kHid * 4));
  return NOMAD_OK;
}

int batch_splits(int B) { return std::max(1, std::min(32, B / 256)); }

// Forward and backward of the batch in S.xb / S.tb (B rows, B a multiple of 64): the gradient of
// the mean squared error with respect to every trainable parameter into S.G (the blob's layout;
// W1's padded input columns get 0), the per-row squared errors into S.se. Mixed precision as in
// the forward pass: BF16 operands of every product (standardised inputs, weights, hidden
// activations, the gradients that flow into a product), FP32 accumulation, FP32 biases and
// output layer; split-K partial sums reduced in a fixed order.
nomad_status batch_gradient(nomad_ctx *ctx, MlpState &S, int B) {
  cudaStream_t s = ctx->stream;
  const int splits = batch_splits(B);
  float *Pm = S.P.as<float>(), *G = S.G.as<float>();
  uint32_t *status = ctx->status.as<uint32_t>();
  k_mlp_forward_tc<false, true><<<(B + kTcRows - 1) / kTcRows, 128, kTcSmem, s>>>(
      S.xb.as<const float>(), B, Pm, S.Wc.as<const unsigned char>(), S.y.as<float>(), status, nomad_res::FeatArgs{},
      FwdSave{S.xbf.as<__nv_bfloat16>(), S.h1.as<__nv_bfloat16>(), S.z1.as<float>(), S.z2.as<float>()});
  k_mse_grad<<<(B + 255) / 256, 256, 0, s>>>(S.y.as<const float>(), S.tb.as<const float>(), B, S.dy.as<float>(),
                                             S.se.as<float>());
  k_dz2<<<(B * kHid + 255) / 256, 256, 0, s>>>(S.dy.as<const float>(), S.z2.as<const float>(), Pm, B,
                                               S.dz2b.as<__nv_bfloat16>(), S.dz2f.as<float>());
  // dw3[c] = sum_r relu(z2[r][c]) * dy[r]; db3 = sum_r dy[r]
  {
    // relu(z2) into dh1, which is free until dH1 below (z2 itself feeds dz2 above)
    float *h2 = S.dh1.as<float>();
    size_t cnt = (size_t)B * kHid;
    k_dz1<<<(unsigned)((cnt + 255) / 256), 256, 0, s>>>(S.z2.as<const float>(), S.z2.as<const float>(), B,
                                                       S.dz1b.as<__nv_bfloat16>(), h2);
    k_colsum<<<1, kHid, 0, s>>>(h2, S.dy.as<const float>(), B, kHid, G + oW3);
    k_colsum<<<1, 1, 0, s>>>(S.dy.as<const float>(), nullptr, B, 1, G + oB3);
  }
  k_colsum<<<1, kHid, 0, s>>>(S.dz2f.as<const float>(), nullptr, B, kHid, G + oB2);
  // dW2[n][k] = sum_i dZ2[i][n] H1[i][k]: A = dZ2^T (stored [B][128]), B = H1 [B][128]
  {
    int kPer = ((B / splits) + kGemmK - 1) / kGemmK * kGemmK;
    int sp = (B + kPer - 1) / kPer;
    dim3 grid(1, 1, sp);
    k_gemm_tc<true, false, kHid><<<grid, 128, 0, s>>>(S.dz2b.as<const __nv_bfloat16>(), S.h1.as<const __nv_bfloat16>(),
                                                      S.part.as<float>(), kHid, kHid, B, kHid, kHid, kPer, status);
    k_reduce_splits<<<64, 256, 0, s>>>(S.part.as<const float>(), sp, (size_t)kHid * kHid, G + oW2);
  }
  // dH1[i][k] = sum_n dZ2[i][n] W2[n][k]: A = dZ2 [B][128], B = W2 [128(n)][128(k)] row-major = [K][N]
  {
    dim3 grid(1, (B + 127) / 128, 1);
    k_gemm_tc<false, false, kHid><<<grid, 128, 0, s>>>(S.dz2b.as<const __nv_bfloat16>(), S.W2b.as<const __nv_bfloat16>(),
                                                       S.dh1.as<float>(), B, kHid, kHid, kHid, kHid, kHid, status);
  }
  k_dz1<<<(B * kHid + 255) / 256, 256, 0, s>>>(S.dh1.as<const float>(), S.z1.as<const float>(), B,
                                               S.dz1b.as<__nv_bfloat16>(), S.dz1f.as<float>());
  k_colsum<<<1, kHid, 0, s>>>(S.dz1f.as<const float>(), nullptr, B, kHid, G + oB1);
  // dW1[n][k] = sum_i dZ1[i][n] X[i][k]: A = dZ1^T, B = Xbf [B][32]
  {
    int kPer = ((B / splits) + kGemmK - 1) / kGemmK * kGemmK;
    int sp = (B + kPer - 1) / kPer;
    dim3 grid(1, 1, sp);
    k_gemm_tc<true, false, kInPad><<<grid, 128, 0, s>>>(S.dz1b.as<const __nv_bfloat16>(), S.xbf.as<const __nv_bfloat16>(),
                                                        S.part.as<float>(), kHid, kInPad, B, kHid, kInPad, kPer, status);
    k_reduce_splits<<<16, 256, 0, s>>>(S.part.as<const float>(), sp, (size_t)kHid * kInPad, G + oW1);
  }
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

}  // namespace

extern "C" nomad_status nomad_mlp_train(nomad_ctx *ctx, const float *features, const float *targets, uint64_t n,
                                        uint32_t steps, uint32_t batch, float lr, float wd, uint64_t seed,
                                        float *loss_out) {
  if (!ctx || !features || !targets || n == 0 || batch == 0 || batch % 64 != 0 || batch > 65536)
    return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "training needs samples and a batch that is a multiple of 64");
  if (n > 0xffffffffull) return nomad_fail(ctx, NOMAD_ERR_LIMIT, "too many samples");
  NOMAD_DEVICE_SCOPE(ctx);
  MlpState &S = mlp(ctx);
  if (!S.ready) {
    nomad_status st = nomad_mlp_init(ctx, seed);
    if (st != NOMAD_OK) return st;
  }
  cudaStream_t s = ctx->stream;
  // Feature statistics (double accumulation on the host), stored in the blob.
  std::vector<double> mean(kIn, 0.0), sq(kIn, 0.0);
  for (uint64_t i = 0; i < n; ++i)
    for (int f = 0; f < kIn; ++f) {
      double v = features[i * kIn + f];
      mean[f] += v;
      sq[f] += v * v;
    }
  float stats[2 * kIn];
  for (int f = 0; f < kIn; ++f) {
    double m = mean[f] / n;
    double var = std::max(0.0, sq[f] / n - m * m);
    stats[f] = (float)m;
    stats[kIn + f] = (float)(1.0 / std::max(std::sqrt(var), 1e-6));
  }
  NOMAD_CUDA(ctx, cudaMemcpyAsync(S.P.as<float>() + oMean, stats, sizeof(stats), cudaMemcpyHostToDevice, s));
  // Every call is a fresh AdamW run from the current weights: the moments start at zero, as the
  // bias correction (from step 1) assumes.
  NOMAD_CUDA(ctx, cudaMemsetAsync(S.M.p, 0, kParams * 4, s));
  NOMAD_CUDA(ctx, cudaMemsetAsync(S.V.p, 0, kParams * 4, s));
  const int B = (int)batch;
  if (S.trainCap < n) {
    NOMAD_CUDA(ctx, S.X.reserve(n * kIn * 4));
    NOMAD_CUDA(ctx, S.T.reserve(n * 4));
    S.trainCap = n;
  }
  NOMAD_CUDA(ctx, cudaMemcpyAsync(S.X.p, features, n * kIn * 4, cudaMemcpyHostToDevice, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(S.T.p, targets, n * 4, cudaMemcpyHostToDevice, s));
  {
    nomad_status st = ensure_batch(ctx, S, B, batch_splits(B));
    if (st != NOMAD_OK) return st;
  }
  std::mt19937_64 rng(seed ^ 0x5EEDull);
  std::vector<uint32_t> perm(n);
  std::iota(perm.begin(), perm.end(), 0u);
  uint64_t cursor = n;
  std::vector<float> se(B);
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float *Pm = S.P.as<float>(), *G = S.G.as<float>();
  for (uint32_t step = 0; step < steps; ++step) {
    if (cursor + B > n) {
      std::shuffle(perm.begin(), perm.end(), rng);
      cursor = 0;
    }
    std::vector<uint32_t> bidx(B);
    for (int i = 0; i < B; ++i) bidx[i] = perm[(cursor + i) % n];
    cursor += B;
    NOMAD_CUDA(ctx, cudaMemcpyAsync(S.idx.p, bidx.data(), (size_t)B * 4, cudaMemcpyHostToDevice, s));
    k_gather<<<(B * kIn + 255) / 256, 256, 0, s>>>(S.X.as<const float>(), S.T.as<const float>(),
                                                   S.idx.as<const uint32_t>(), B, S.xb.as<float>(), S.tb.as<float>());
    nomad_status st = batch_gradient(ctx, S, B);
    if (st != NOMAD_OK) return st;
    float bc1 = 1.0f - std::pow(b1, (float)(step + 1)), bc2 = 1.0f - std::pow(b2, (float)(step + 1));
    k_adamw<<<(oMean + 255) / 256, 256, 0, s>>>(Pm, G, S.M.as<float>(), S.V.as<float>(), oMean, lr, b1, b2, eps, wd,
                                                bc1, bc2);
    st = refresh(ctx, S);
    if (st != NOMAD_OK) return st;
    NOMAD_CUDA(ctx, cudaGetLastError());
    if (loss_out) {
      NOMAD_CUDA(ctx, cudaMemcpyAsync(se.data(), S.se.p, (size_t)B * 4, cudaMemcpyDeviceToHost, s));
      NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
      double acc = 0.0;
      for (int i = 0; i < B; ++i) acc += se[i];
      loss_out[step] = (float)(acc / B);
    }
  }
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_mlp_gradient(nomad_ctx *ctx, const float *features, const float *targets, uint64_t n,
                                           float *grad, float *loss) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!features || !targets || !grad || n == 0 || n % 64 != 0 || n > 65536)
    return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "the gradient needs 64 to 65,536 samples, a multiple of 64");
  NOMAD_DEVICE_SCOPE(ctx);
  MlpState &S = mlp(ctx);
  if (!S.ready) return nomad_fail(ctx, NOMAD_ERR_NOT_READY, "MLP not initialised or trained");
  const int B = (int)n;
  nomad_status st = ensure_batch(ctx, S, B, batch_splits(B));
  if (st != NOMAD_OK) return st;
  cudaStream_t s = ctx->stream;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(S.xb.p, features, n * kIn * 4, cudaMemcpyHostToDevice, s));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(S.tb.p, targets, n * 4, cudaMemcpyHostToDevice, s));
  NOMAD_CUDA(ctx, cudaMemsetAsync(S.G.p, 0, kParams * 4, s));
  st = batch_gradient(ctx, S, B);
  if (st != NOMAD_OK) return st;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(grad, S.G.p, kParams * 4, cudaMemcpyDeviceToHost, s));
  std::vector<float> se(B);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(se.data(), S.se.p, (size_t)B * 4, cudaMemcpyDeviceToHost, s));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(s));
  if (loss) {
    double acc = 0.0;
    for (int i = 0; i < B; ++i) acc += se[i];
    *loss = (float)(acc / B);
  }
  return NOMAD_OK;
}
