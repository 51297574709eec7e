// Residency compaction of the SceneBVH arrays on the device.
//
// Produces, from the full SceneBVH arrays and a per-primitive active mask, exactly the compacted
// arrays the reference's rebuildResidentResources builds on the host when residency compaction
// is on (Nomad Path Tracer/Renderer/Renderer.cpp:5359-5560, the cached-BLAS path): active
// primitives in object order and, within an object, in BLAS leaf order; each object's BLAS
// pruned of leaves without active primitives, inner nodes with one surviving child replaced by
// that child, surviving nodes numbered in post-order (children before parents) with unchanged
// bounds; instance records pointing at the compact ranges; the TLAS unchanged.
//
// The reference walks each object's tree recursively. Here every primitive and every node is
// one thread, with two exclusive scans:
//   * cpos = exclusive scan of the active flags in leaf order. A primitive's compact index is
//     cpos at its leaf position; a leaf keeps cpos[first] and cpos[end] - cpos[first] primitives.
//     Because a SceneBVH subtree covers a contiguous leaf range (left subtree first), a subtree
//     survives iff its range holds an active primitive, and an inner node is emitted iff both
//     children survive (otherwise it is dropped or replaced by its surviving child).
//   * epos = exclusive scan of the emitted flags in node (pre-)order. A node's post-order index
//     among emitted nodes is epos[end of its subtree] - 1 - (emitted strict ancestors), its right
//     child's representative is the node just before it, and its left child's representative
//     precedes the right subtree's emitted nodes.
// Every pointer walk is bounded by the traversal stack limit and every index is range-checked;
// a violation sets a bit in counts[2] instead of faulting.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "../../../include/nomad_scene.h"

namespace {

constexpr int kT = 256;           // threads per block of the per-item kernels
constexpr int kScanT = 1024;      // threads per scan block
constexpr int kScanPer = 4;       // items per scan thread
constexpr int kScanTile = kScanT * kScanPer;
constexpr int kMaxWalk = 128;     // longest root-to-leaf walk accepted

enum : uint32_t { kErrIndex = 1u, kErrDepth = 2u, kErrLayout = 4u };

__device__ __forceinline__ int32_t left_first(const float4 *bvh, int32_t i) {
  return __float_as_int(__ldg(&bvh[2 * (size_t)i].w));
}
__device__ __forceinline__ int32_t count_of(const float4 *bvh, int32_t i) {
  return __float_as_int(__ldg(&bvh[2 * (size_t)i + 1].w));
}

__device__ __forceinline__ void flag(uint32_t *err, uint32_t bit) { atomicOr(err, bit); }

// ---- exclusive scan of u32 flags (reduce, scan of tile sums, down-sweep) ----

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t t = __shfl_up_sync(0xffffffffu, v, d);
    if (lane >= d) v += t;
  }
  return v;
}

// Exclusive prefix of v over the block; *total receives the block sum.
__device__ uint32_t block_exclusive(uint32_t v, uint32_t *sh, uint32_t *total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint32_t inc = warp_inclusive(v);
  if (lane == 31) sh[w] = inc;
  __syncthreads();
  if (w == 0) {
    const uint32_t s = lane < nw ? sh[lane] : 0u;
    const uint32_t si = warp_inclusive(s);
    if (lane < nw) sh[lane] = si;
  }
  __syncthreads();
  const uint32_t off = w ? sh[w - 1] : 0u;
  *total = sh[nw - 1];
  __syncthreads();
  return off + inc - v;
}

__global__ void __launch_bounds__(kScanT) k_scan_reduce(const uint32_t *__restrict__ f, uint32_t m,
                                                        uint32_t *__restrict__ sums) {
  __shared__ uint32_t sh[32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
  uint32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k)
    if (base + k < m) s += f[base + k];
  uint32_t tot;
  block_exclusive(s, sh, &tot);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block: exclusive scan of the tile sums in place; pos[m] = total.
__global__ void __launch_bounds__(kScanT) k_scan_top(uint32_t *__restrict__ sums, uint32_t tiles,
                                                     uint32_t *__restrict__ pos, uint32_t m) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (uint32_t b = 0; b < tiles; b += kScanT) {
    const uint32_t i = b + threadIdx.x;
    const uint32_t v = i < tiles ? sums[i] : 0u;
    uint32_t tot;
    const uint32_t ex = block_exclusive(v, sh, &tot);
    if (i < tiles) sums[i] = carry + ex;
    carry += tot;
  }
  if (threadIdx.x == 0) pos[m] = carry;
}

__global__ void __launch_bounds__(kScanT) k_scan_down(const uint32_t *__restrict__ f, uint32_t m,
                                                      const uint32_t *__restrict__ sums, uint32_t *__restrict__ pos) {
  __shared__ uint32_t sh[32];
  const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanPer;
  uint32_t v[kScanPer], s = 0;
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    v[k] = base + k < m ? f[base + k] : 0u;
    s += v[k];
  }
  uint32_t tot;
  uint32_t run = sums[blockIdx.x] + block_exclusive(s, sh, &tot);
#pragma unroll
  for (int k = 0; k < kScanPer; ++k) {
    if (base + k < m) pos[base + k] = run;
    run += v[k];
  }
}

// ---- compaction ----

// Leaf-order activity: a[j] = active[primIdx[j]].
__global__ void k_prim_flags(const int32_t *__restrict__ primIdx, const uint8_t *__restrict__ active, uint32_t n,
                             uint32_t *__restrict__ a, uint32_t *__restrict__ err) {
  const uint32_t j = blockIdx.x * kT + threadIdx.x;
  if (j >= n) return;
  const int32_t g = primIdx[j];
  if (g < 0 || (uint32_t)g >= n) {
    flag(err, kErrIndex);
    a[j] = 0;
    return;
  }
  a[j] = active[g] ? 1u : 0u;
}

// Active primitives to their compact slots: remap (compact -> global), compact primitive index
// (its own slot), global -> compact map.
__global__ void k_gather(const int32_t *__restrict__ primIdx, const uint32_t *__restrict__ a,
                         const uint32_t *__restrict__ cpos, uint32_t n, uint32_t *__restrict__ oRemap,
                         int32_t *__restrict__ oIdx, int32_t *__restrict__ oPrimToRes) {
  const uint32_t j = blockIdx.x * kT + threadIdx.x;
  if (j >= n) return;
  const int32_t g = primIdx[j];
  const bool on = a[j] != 0;  // only valid indices are flagged
  const uint32_t k = cpos[j];
  if (g >= 0 && (uint32_t)g < n) oPrimToRes[g] = on ? (int32_t)k : -1;
  if (on) {
    oRemap[k] = (uint32_t)g;
    oIdx[k] = (int32_t)k;
  }
}

// The active primitives' packed primitive (7 float4) and material (5 float4), one float4 per
// thread in compact order: reads follow the remap, writes are contiguous.
__global__ void __launch_bounds__(kT) k_copy_prims(const uint32_t *__restrict__ remap, const uint32_t *__restrict__ count,
                                                   const float4 *__restrict__ prims, const float4 *__restrict__ mats,
                                                   float4 *__restrict__ oPrims, float4 *__restrict__ oMats) {
  const unsigned long long items = (unsigned long long)(*count) * 12ull;
  for (unsigned long long t = (unsigned long long)blockIdx.x * kT + threadIdx.x; t < items;
       t += (unsigned long long)gridDim.x * kT) {
    const unsigned long long k = t / 12ull;
    const uint32_t part = (uint32_t)(t - k * 12ull);
    const uint32_t g = __ldg(&remap[k]);
    if (part < 7u) oPrims[k * 7 + part] = __ldg(&prims[(size_t)g * 7 + part]);
    else oMats[k * 5 + (part - 7u)] = __ldg(&mats[(size_t)g * 5 + (part - 7u)]);
  }
}

// First leaf position covered by the subtree of node u (walk left children to a leaf).
__device__ __forceinline__ bool leftmost_start(const float4 *bvh, uint32_t N, int32_t u, int32_t &start,
                                               uint32_t *err) {
  for (int s = 0; s < kMaxWalk; ++s) {
    if (u < 0 || (uint32_t)u >= N) {
      flag(err, kErrIndex);
      return false;
    }
    const int32_t c = count_of(bvh, u), lf = left_first(bvh, u);
    if (c > 0) {
      start = lf;
      return true;
    }
    u = lf;
  }
  flag(err, kErrDepth);
  return false;
}

// Last node (a leaf, in pre-order) of the subtree of node u; its index + 1 ends the subtree.
__device__ __forceinline__ bool rightmost_leaf(const float4 *bvh, uint32_t N, int32_t u, int32_t &leaf,
                                               uint32_t *err) {
  for (int s = 0; s < kMaxWalk; ++s) {
    if (u < 0 || (uint32_t)u >= N) {
      flag(err, kErrIndex);
      return false;
    }
    const int32_t c = count_of(bvh, u);
    if (c > 0) {
      leaf = u;
      return true;
    }
    u = -c;
  }
  flag(err, kErrDepth);
  return false;
}

// Node flags: bit 0 emitted, bit 1 survives; e[v] = emitted for the scan.
__global__ void k_node_flags(const float4 *__restrict__ bvh, uint32_t N, const uint32_t *__restrict__ cpos,
                             uint32_t n, uint8_t *__restrict__ nflag, uint32_t *__restrict__ e,
                             uint32_t *__restrict__ err) {
  const uint32_t v = blockIdx.x * kT + threadIdx.x;
  if (v >= N) return;
  const int32_t c = count_of(bvh, v), lf = left_first(bvh, v);
  uint8_t fl = 0;
  if (c > 0) {
    if (lf < 0 || (int64_t)lf + c > (int64_t)n) {
      flag(err, kErrIndex);
    } else if (cpos[lf + c] != cpos[lf]) {
      fl = 3;
    }
  } else {
    int32_t s = 0, mid = 0, rl = 0;
    if (leftmost_start(bvh, N, lf, s, err) && leftmost_start(bvh, N, -c, mid, err) &&
        rightmost_leaf(bvh, N, -c, rl, err)) {
      const int64_t end = (int64_t)left_first(bvh, rl) + count_of(bvh, rl);
      if (s < 0 || mid < s || end < mid || end > (int64_t)n) {
        flag(err, kErrLayout);
      } else {
        const bool kl = cpos[mid] != cpos[s], kr = cpos[end] != cpos[mid];
        fl = (uint8_t)((kl && kr ? 1 : 0) | (kl || kr ? 2 : 0));
      }
    }
  }
  nflag[v] = fl;
  e[v] = fl & 1u;
}

// Subtree of each object: root[v] for every node of the object's range. One block per object.
__global__ void k_node_roots(const float4 *__restrict__ bvh, uint32_t N, const nomad_instance_record *__restrict__ inst,
                             uint32_t nobj, int32_t *__restrict__ rootOf, int32_t *__restrict__ objEnd,
                             uint32_t *__restrict__ err) {
  const uint32_t o = blockIdx.x;
  if (o >= nobj) return;
  const int32_t r = inst[o].blas_root_index;
  __shared__ int32_t sEnd;
  if (threadIdx.x == 0) {
    int32_t leaf = -1;
    sEnd = (r >= 0 && rightmost_leaf(bvh, N, r, leaf, err)) ? leaf + 1 : -1;
    objEnd[o] = sEnd;
  }
  __syncthreads();
  if (sEnd < 0) return;
  for (int32_t v = r + (int32_t)threadIdx.x; v < sEnd; v += (int32_t)blockDim.x) rootOf[v] = r;
}

// Emitted nodes to their post-order slots.
__global__ void k_emit(const float4 *__restrict__ bvh, uint32_t N, const uint32_t *__restrict__ cpos,
                       const uint8_t *__restrict__ nflag, const uint32_t *__restrict__ epos,
                       const int32_t *__restrict__ rootOf, float4 *__restrict__ oBvh, uint32_t *__restrict__ err) {
  const int32_t v = (int32_t)(blockIdx.x * kT + threadIdx.x);
  if ((uint32_t)v >= N || !(nflag[v] & 1u)) return;
  // emitted strict ancestors: walk down from the object's root
  int32_t u = rootOf[v];
  uint32_t anc = 0;
  int s = 0;
  for (; s < kMaxWalk && u != v; ++s) {
    if (u < 0 || (uint32_t)u >= N || u > v) {
      flag(err, kErrLayout);
      return;
    }
    if (nflag[u] & 1u) ++anc;
    const int32_t c = count_of(bvh, u);
    if (c > 0) {
      flag(err, kErrLayout);
      return;
    }
    u = v < -c ? left_first(bvh, u) : -c;
  }
  if (u != v) {
    flag(err, kErrDepth);
    return;
  }
  const int32_t c = count_of(bvh, v), lf = left_first(bvh, v);
  int32_t end = v + 1;
  if (c <= 0) {
    int32_t rl = 0;
    if (!rightmost_leaf(bvh, N, -c, rl, err)) return;
    end = rl + 1;
  }
  const int32_t P = (int32_t)(epos[end] - 1u - anc);
  float4 lo = __ldg(&bvh[2 * (size_t)v]), hi = __ldg(&bvh[2 * (size_t)v + 1]);
  if (c > 0) {
    lo.w = __int_as_float((int32_t)cpos[lf]);
    hi.w = __int_as_float((int32_t)(cpos[lf + c] - cpos[lf]));
  } else {
    const int32_t rightRep = P - 1;
    const int32_t leftRep = rightRep - (int32_t)(epos[end] - epos[-c]);
    lo.w = __int_as_float(leftRep);
    hi.w = __int_as_float(-rightRep);
  }
  oBvh[2 * (size_t)P] = lo;
  oBvh[2 * (size_t)P + 1] = hi;
}

__global__ void k_records(const nomad_instance_record *__restrict__ inst, uint32_t nobj, uint32_t n,
                          const uint32_t *__restrict__ cpos, const uint32_t *__restrict__ epos, uint32_t N,
                          const int32_t *__restrict__ objEnd, nomad_instance_record *__restrict__ oInst,
                          uint32_t *__restrict__ counts, uint32_t *__restrict__ err) {
  const uint32_t o = blockIdx.x * kT + threadIdx.x;
  if (o == 0) {
    counts[0] = cpos[n];
    counts[1] = epos[N];
  }
  if (o >= nobj) return;
  const nomad_instance_record r = inst[o];
  const uint64_t first = r.primitive_index_base, end = first + r.primitive_count;
  nomad_instance_record w;
  w.blas_root_index = -1;
  if (end > n || r.primitive_base != r.primitive_index_base) {
    flag(err, kErrIndex);
    w.primitive_base = w.primitive_index_base = 0;
    w.primitive_count = 0;
    oInst[o] = w;
    return;
  }
  const uint32_t base = cpos[first], cnt = cpos[end] - base;
  w.primitive_base = base;
  w.primitive_index_base = base;
  w.primitive_count = cnt;
  if (cnt > 0) {
    const int32_t root = r.blas_root_index, oe = root >= 0 ? objEnd[o] : -1;
    if (root < 0 || oe <= root || epos[oe] == epos[root])
      flag(err, kErrLayout);  // active primitives without a BLAS over them
    else
      w.blas_root_index = (int32_t)(epos[oe] - 1u);  // the pruned root is last in post-order
  }
  oInst[o] = w;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

struct Work {
  uint32_t *a, *cpos, *e, *epos, *sums, *err;
  uint8_t *nflag;
  int32_t *rootOf, *objEnd;
};

size_t layout(uint32_t n, uint32_t N, uint32_t nobj, char *base, Work *w) {
  const size_t tiles = ((size_t)(n > N ? n : N) + kScanTile - 1) / kScanTile + 1;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char *p = base ? base + off : nullptr;
    off += align_up(bytes);
    return p;
  };
  char *a = take((size_t)n * 4), *cpos = take(((size_t)n + 1) * 4), *e = take((size_t)N * 4),
       *epos = take(((size_t)N + 1) * 4), *sums = take(tiles * 4), *err = take(4), *nflag = take(N),
       *rootOf = take((size_t)N * 4), *objEnd = take((size_t)nobj * 4);
  if (w) {
    w->a = (uint32_t *)a;
    w->cpos = (uint32_t *)cpos;
    w->e = (uint32_t *)e;
    w->epos = (uint32_t *)epos;
    w->sums = (uint32_t *)sums;
    w->err = (uint32_t *)err;
    w->nflag = (uint8_t *)nflag;
    w->rootOf = (int32_t *)rootOf;
    w->objEnd = (int32_t *)objEnd;
  }
  return off;
}

cudaError_t scan(const uint32_t *f, uint32_t m, uint32_t *sums, uint32_t *pos, cudaStream_t s) {
  const uint32_t tiles = (m + kScanTile - 1) / kScanTile;
  if (tiles) k_scan_reduce<<<tiles, kScanT, 0, s>>>(f, m, sums);
  k_scan_top<<<1, kScanT, 0, s>>>(sums, tiles, pos, m);
  if (tiles) k_scan_down<<<tiles, kScanT, 0, s>>>(f, m, sums, pos);
  return cudaGetLastError();
}

}  // namespace

extern "C" size_t nomad_compact_workspace_bytes(uint32_t prim_count, uint32_t bvh_node_count,
                                                uint32_t object_count) {
  return layout(prim_count, bvh_node_count, object_count, nullptr, nullptr);
}

extern "C" nomad_status nomad_scenebvh_compact_gpu(const nomad_scenebvh_device *in, const uint8_t *prim_active,
                                                   void *workspace, size_t workspace_bytes,
                                                   const nomad_compact_out *out, void *stream) {
  if (!in || !out || !prim_active || !workspace) return NOMAD_ERR_INVALID_ARGUMENT;
  const uint32_t n = in->prim_count, N = in->bvh_node_count, nobj = in->object_count;
  if (n == 0 || nobj == 0 || !in->bvh_nodes || !in->prims || !in->materials || !in->prim_indices ||
      !in->instances || !out->bvh_nodes || !out->prims || !out->materials || !out->prim_indices ||
      !out->remap || !out->prim_to_resident || !out->instances || !out->counts)
    return NOMAD_ERR_INVALID_ARGUMENT;
  if (n > 0x7fffffffu || N > 0x7fffffffu) return NOMAD_ERR_LIMIT;
  Work w;
  if (workspace_bytes < layout(n, N, nobj, static_cast<char *>(workspace), &w)) return NOMAD_ERR_INVALID_ARGUMENT;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const float4 *bvh = reinterpret_cast<const float4 *>(in->bvh_nodes);
  const unsigned gp = (n + kT - 1) / kT, gn = (N + kT - 1) / kT;
  if (cudaMemsetAsync(w.err, 0, 4, s) != cudaSuccess) return NOMAD_ERR_CUDA;
  if (N && cudaMemsetAsync(w.rootOf, 0xff, (size_t)N * 4, s) != cudaSuccess) return NOMAD_ERR_CUDA;
  k_prim_flags<<<gp, kT, 0, s>>>(in->prim_indices, prim_active, n, w.a, w.err);
  if (scan(w.a, n, w.sums, w.cpos, s) != cudaSuccess) return NOMAD_ERR_CUDA;
  k_gather<<<gp, kT, 0, s>>>(in->prim_indices, w.a, w.cpos, n, out->remap, out->prim_indices, out->prim_to_resident);
  {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned gc = (unsigned)std::min<uint64_t>((uint64_t)sms * 16, ((uint64_t)n * 12 + kT - 1) / kT);
    k_copy_prims<<<gc, kT, 0, s>>>(out->remap, w.cpos + n, reinterpret_cast<const float4 *>(in->prims),
                                   reinterpret_cast<const float4 *>(in->materials),
                                   reinterpret_cast<float4 *>(out->prims), reinterpret_cast<float4 *>(out->materials));
  }
  if (N) {
    k_node_flags<<<gn, kT, 0, s>>>(bvh, N, w.cpos, n, w.nflag, w.e, w.err);
    k_node_roots<<<nobj, kT, 0, s>>>(bvh, N, in->instances, nobj, w.rootOf, w.objEnd, w.err);
  } else {
    if (cudaMemsetAsync(w.objEnd, 0xff, (size_t)nobj * 4, s) != cudaSuccess) return NOMAD_ERR_CUDA;
  }
  if (scan(w.e, N, w.sums, w.epos, s) != cudaSuccess) return NOMAD_ERR_CUDA;
  if (N)
    k_emit<<<gn, kT, 0, s>>>(bvh, N, w.cpos, w.nflag, w.epos, w.rootOf, reinterpret_cast<float4 *>(out->bvh_nodes),
                             w.err);
  k_records<<<(nobj + kT - 1) / kT, kT, 0, s>>>(in->instances, nobj, n, w.cpos, w.epos, N, w.objEnd, out->instances,
                                                 out->counts, w.err);
  if (cudaMemcpyAsync(out->counts + 2, w.err, 4, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return NOMAD_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? NOMAD_OK : NOMAD_ERR_CUDA;
}
