// SceneBVH BLAS construction on the GPU, bit-identical to the host builder (host/scenebvh.cpp,
// itself restated from Scene::buildBVHRecursive / evaluateSAHSplit, Nomad Path Tracer/Scene/
// SceneBVH.cpp:549-623 and :704-815).
//
// The recursion becomes a level-synchronous loop: every node of a level (of every object) is one
// task, one block per task. A block
//   1. reduces its primitives' bounds in primitive order (ties keep the first value, as the
//      host's running min/max does, so even the sign of a zero bound matches),
//   2. stops at <= 8 primitives or a zero-area box (a leaf),
//   3. bins centroids into 12 bins per axis (counts and bin bounds by shared-memory atomics: bin
//      bounds only feed surface areas, where the sign of a zero cannot matter) and evaluates the
//      SAH exactly as the host does, in one thread, in the same operation order,
//   4. stable-sorts its index range by the split axis centroid (a bitonic sort of (key, position)
//      pairs in shared memory up to 2,048 primitives, a block LSD radix sort with a stable tile
//      scatter beyond), and appends its two children to the next level.
// Task ids link parents to children; the host then numbers each object's nodes in pre-order,
// which is the order the recursive builder emits, and hands the result to the shared finishing
// stage (concatenation, TLAS, packing). Float keys map -0.0 to +0.0 so the sorts order equal
// centroids like the host comparator (a < b) does.
#include <cuda_runtime.h>

#include <algorithm>
#include <limits>
#include <memory>
#include <new>
#include <vector>

#include "../../../include/nomad_scene.h"
#include "../host/scenebvh_internal.h"
#include "device_scope.h"

namespace {

constexpr int kB = 256;           // threads per task block
constexpr int kBins = 12;
constexpr int kSmallSort = 2048;  // ranges sorted in shared memory
constexpr float kFmax = std::numeric_limits<float>::max();

struct Task {
  int32_t start, count, obj, pad;
};

struct TaskOut {
  float mn[3], mx[3];
  int32_t left, right;  // child task ids, -1 for a leaf
};

// Float <-> int with the same order (for shared-memory atomic min / max).
__device__ __forceinline__ int f2o(float f) {
  int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7fffffff); }

// Ascending-order key of a float with -0.0 equal to +0.0.
__device__ __forceinline__ uint32_t fkey(float f) {
  if (f == 0.0f) f = 0.0f;
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// Per primitive (original index): bounds and the centroid used for binning and sorting
// (primitiveBounds SceneBVH.cpp:843-864, primitiveAxisValue :822-830).
__global__ void k_prim_info(const int32_t *__restrict__ type, const float *__restrict__ geom, uint32_t n,
                            float *__restrict__ info) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const float *g = geom + (size_t)p * NOMAD_PRIM_GEOM_FLOATS;
  float mn[3], mx[3], c[3];
  const int t = type[p];
  if (t == NOMAD_PRIM_SPHERE) {
    const float r = g[3];
    for (int k = 0; k < 3; ++k) {
      mn[k] = g[k] - r;
      mx[k] = g[k] + r;
      c[k] = g[k];
    }
  } else if (t == NOMAD_PRIM_RECTANGLE) {
    for (int k = 0; k < 3; ++k) {
      const float ck = g[k], e1 = g[3 + k], e2 = g[6 + k];
      const float c1 = ck - e1 - e2, c2 = ck - e1 + e2, c3 = ck + e1 - e2, c4 = ck + e1 + e2;
      const float m12 = c2 < c1 ? c2 : c1, m34 = c4 < c3 ? c4 : c3;
      const float x12 = c1 < c2 ? c2 : c1, x34 = c3 < c4 ? c4 : c3;
      mn[k] = m34 < m12 ? m34 : m12;
      mx[k] = x12 < x34 ? x34 : x12;
      c[k] = ck;
    }
  } else {
    for (int k = 0; k < 3; ++k) {
      const float a = g[k], b = g[3 + k], cc = g[6 + k];
      const float mbc = cc < b ? cc : b, xbc = b < cc ? cc : b;
      mn[k] = mbc < a ? mbc : a;
      mx[k] = a < xbc ? xbc : a;
      c[k] = (a + b + cc) / 3.0f;
    }
  }
  float *o = info + (size_t)p * 9;
  for (int k = 0; k < 3; ++k) {
    o[k] = mn[k];
    o[3 + k] = mx[k];
    o[6 + k] = c[k];
  }
}

// (value, position) reductions keeping the first position among equal values.
struct VP {
  float v;
  int p;
};
__device__ __forceinline__ VP vp_min(VP a, VP b) { return (b.v < a.v || (b.v == a.v && b.p < a.p)) ? b : a; }
__device__ __forceinline__ VP vp_max(VP a, VP b) { return (a.v < b.v || (b.v == a.v && b.p < a.p)) ? b : a; }

__device__ VP block_vp(VP x, bool isMin, VP *sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = 16; d > 0; d >>= 1) {
    VP y{__shfl_down_sync(0xffffffffu, x.v, d), __shfl_down_sync(0xffffffffu, x.p, d)};
    x = isMin ? vp_min(x, y) : vp_max(x, y);
  }
  if (lane == 0) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    x = lane < kB / 32 ? sh[lane] : VP{isMin ? kFmax : -kFmax, INT32_MAX};
    for (int d = 16; d > 0; d >>= 1) {
      VP y{__shfl_down_sync(0xffffffffu, x.v, d), __shfl_down_sync(0xffffffffu, x.p, d)};
      x = isMin ? vp_min(x, y) : vp_max(x, y);
    }
    if (lane == 0) sh[0] = x;
  }
  __syncthreads();
  const VP r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ float surface_area(const float mn[3], const float mx[3]) {
  const float dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct LevelArgs {
  const float *info;      // 9 floats per primitive
  int32_t *idx;           // primitive permutation (primitiveIndices)
  int32_t *tmpIdx;        // radix scatter buffer, same positions as idx
  uint32_t *keyA, *keyB;  // radix keys
  Task *tasks;
  TaskOut *out;
  uint32_t *taskCount;
  uint32_t lo, hi;        // this level's task ids
};

__global__ void __launch_bounds__(kB) k_build_level(LevelArgs A) {
  __shared__ VP red[kB / 32];
  __shared__ int cbound[6];                 // centroid min xyz, max xyz (ordered ints)
  __shared__ int binCnt[3][kBins];
  __shared__ int binB[3][kBins][6];         // ordered ints: min xyz, max xyz
  __shared__ int decision[2];               // axis, left count (or -1 for a leaf)
  __shared__ unsigned long long comp[kSmallSort];
  __shared__ int oldIdx[kSmallSort];
  __shared__ int hist[256], binStart[256], run[256];
  __shared__ int wcnt[kB / 32][257];

  for (uint32_t tid = A.lo + blockIdx.x; tid < A.hi; tid += gridDim.x) {
    const Task T = A.tasks[tid];
    const int s = T.start, count = T.count, t = threadIdx.x;
    // 1. node bounds in primitive order, first value kept on ties
    VP lo3[3], hi3[3];
    for (int k = 0; k < 3; ++k) {
      lo3[k] = VP{kFmax, INT32_MAX};
      hi3[k] = VP{-kFmax, INT32_MAX};
    }
    for (int i = t; i < count; i += kB) {
      const float *f = A.info + (size_t)A.idx[s + i] * 9;
      for (int k = 0; k < 3; ++k) {
        lo3[k] = vp_min(lo3[k], VP{f[k], i});
        hi3[k] = vp_max(hi3[k], VP{f[3 + k], i});
      }
    }
    float bmn[3], bmx[3];
    for (int k = 0; k < 3; ++k) {
      bmn[k] = block_vp(lo3[k], true, red).v;
      bmx[k] = block_vp(hi3[k], false, red).v;
    }
    if (t == 0) {
      TaskOut &o = A.out[tid];
      for (int k = 0; k < 3; ++k) {
        o.mn[k] = bmn[k];
        o.mx[k] = bmx[k];
      }
      o.left = o.right = -1;
    }
    const float parentArea = surface_area(bmn, bmx);
    if (count <= 8 || parentArea <= 0.0f) continue;  // uniform across the block
    // 2. centroid bounds and bins
    if (t < 3) {
      cbound[t] = f2o(kFmax);
      cbound[3 + t] = f2o(-kFmax);
    }
    for (int e = t; e < 3 * kBins; e += kB) {
      const int a = e / kBins, b = e % kBins;
      binCnt[a][b] = 0;
      for (int k = 0; k < 3; ++k) {
        binB[a][b][k] = f2o(kFmax);
        binB[a][b][3 + k] = f2o(-kFmax);
      }
    }
    __syncthreads();
    for (int i = t; i < count; i += kB) {
      const float *f = A.info + (size_t)A.idx[s + i] * 9;
      for (int k = 0; k < 3; ++k) {
        atomicMin(&cbound[k], f2o(f[6 + k]));
        atomicMax(&cbound[3 + k], f2o(f[6 + k]));
      }
    }
    __syncthreads();
    float clo[3], chi[3];
    for (int k = 0; k < 3; ++k) {
      clo[k] = o2f(cbound[k]);
      chi[k] = o2f(cbound[3 + k]);
    }
    for (int i = t; i < count; i += kB) {
      const float *f = A.info + (size_t)A.idx[s + i] * 9;
      for (int a = 0; a < 3; ++a) {
        const float range = chi[a] - clo[a];
        if (range <= 1e-6f) continue;
        const float inv = 1.0f / range;
        int bin = (int)((f[6 + a] - clo[a]) * inv * (float)kBins);
        bin = max(0, min(kBins - 1, bin));
        atomicAdd(&binCnt[a][bin], 1);
        for (int k = 0; k < 3; ++k) {
          atomicMin(&binB[a][bin][k], f2o(f[k]));
          atomicMax(&binB[a][bin][3 + k], f2o(f[3 + k]));
        }
      }
    }
    __syncthreads();
    // 3. SAH, exactly as the host evaluates it
    if (t == 0) {
      int bestAxis = -1, bestLeft = 0;
      float bestCost = kFmax;
      for (int a = 0; a < 3; ++a) {
        const float range = chi[a] - clo[a];
        if (range <= 1e-6f) continue;
        float pmn[kBins][3], pmx[kBins][3], smn[kBins][3], smx[kBins][3];
        int pc[kBins], sc[kBins];
        float rmn[3] = {kFmax, kFmax, kFmax}, rmx[3] = {-kFmax, -kFmax, -kFmax};
        int rc = 0;
        for (int i = 0; i < kBins; ++i) {
          if (binCnt[a][i] > 0)
            for (int k = 0; k < 3; ++k) {
              const float bn = o2f(binB[a][i][k]), bx = o2f(binB[a][i][3 + k]);
              rmn[k] = bn < rmn[k] ? bn : rmn[k];
              rmx[k] = rmx[k] < bx ? bx : rmx[k];
            }
          rc += binCnt[a][i];
          for (int k = 0; k < 3; ++k) {
            pmn[i][k] = rmn[k];
            pmx[i][k] = rmx[k];
          }
          pc[i] = rc;
        }
        for (int k = 0; k < 3; ++k) {
          rmn[k] = kFmax;
          rmx[k] = -kFmax;
        }
        rc = 0;
        for (int i = kBins - 1; i >= 0; --i) {
          if (binCnt[a][i] > 0)
            for (int k = 0; k < 3; ++k) {
              const float bn = o2f(binB[a][i][k]), bx = o2f(binB[a][i][3 + k]);
              rmn[k] = bn < rmn[k] ? bn : rmn[k];
              rmx[k] = rmx[k] < bx ? bx : rmx[k];
            }
          rc += binCnt[a][i];
          for (int k = 0; k < 3; ++k) {
            smn[i][k] = rmn[k];
            smx[i][k] = rmx[k];
          }
          sc[i] = rc;
        }
        for (int i = 0; i < kBins - 1; ++i) {
          const int l = pc[i], r = sc[i + 1];
          if (l == 0 || r == 0) continue;
          const float saL = surface_area(pmn[i], pmx[i]);
          const float saR = surface_area(smn[i + 1], smx[i + 1]);
          const float cost = 0.125f + (saL / parentArea) * l + (saR / parentArea) * r;
          if (cost < bestCost) {
            bestCost = cost;
            bestAxis = a;
            bestLeft = l;
          }
        }
      }
      int leftCount = bestAxis == -1 ? count / 2 : min(bestLeft, count - 1);
      if (bestAxis == -1 || leftCount == 0 || leftCount >= count) leftCount = -1;
      decision[0] = bestAxis;
      decision[1] = leftCount;
    }
    __syncthreads();
    const int axis = decision[0], leftCount = decision[1];
    if (leftCount < 0) continue;  // a leaf
    // 4. stable sort of the range by the axis centroid
    if (count <= kSmallSort) {
      int n2 = 1;
      while (n2 < count) n2 <<= 1;
      for (int i = t; i < n2; i += kB) {
        if (i < count) {
          const int p = A.idx[s + i];
          oldIdx[i] = p;
          comp[i] = ((unsigned long long)fkey(A.info[(size_t)p * 9 + 6 + axis]) << 32) | (unsigned)i;
        } else {
          comp[i] = ~0ull;
        }
      }
      __syncthreads();
      for (int k = 2; k <= n2; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
          for (int i = t; i < n2; i += kB) {
            const int l = i ^ j;
            if (l > i) {
              const unsigned long long a = comp[i], b = comp[l];
              if ((a > b) == ((i & k) == 0)) {
                comp[i] = b;
                comp[l] = a;
              }
            }
          }
          __syncthreads();
        }
      for (int i = t; i < count; i += kB) A.idx[s + i] = oldIdx[(int)(comp[i] & 0xffffffffu)];
      __syncthreads();
    } else {
      // LSD radix sort over 4 digits; positions [s, s + count) of keyA/keyB and idx/tmpIdx
      for (int i = t; i < count; i += kB) A.keyA[s + i] = fkey(A.info[(size_t)A.idx[s + i] * 9 + 6 + axis]);
      for (int e = t; e < (kB / 32) * 257; e += kB) (&wcnt[0][0])[e] = 0;
      __syncthreads();
      const int lane = t & 31, warp = t >> 5;
      for (int pass = 0; pass < 4; ++pass) {
        const uint32_t *ks = (pass & 1) ? A.keyB : A.keyA;
        uint32_t *kd = (pass & 1) ? A.keyA : A.keyB;
        const int32_t *is = (pass & 1) ? A.tmpIdx : A.idx;
        int32_t *id = (pass & 1) ? A.idx : A.tmpIdx;
        const int shift = 8 * pass;
        hist[t] = 0;
        run[t] = 0;
        __syncthreads();
        for (int i = t; i < count; i += kB) atomicAdd(&hist[(ks[s + i] >> shift) & 255], 1);
        __syncthreads();
        if (t == 0) {
          int acc = 0;
          for (int d = 0; d < 256; ++d) {
            binStart[d] = acc;
            acc += hist[d];
          }
        }
        __syncthreads();
        for (int base = 0; base < count; base += kB) {
          const int i = base + t;
          const bool has = i < count;
          const uint32_t key = has ? ks[s + i] : 0u;
          const int32_t val = has ? is[s + i] : 0;
          const int d = has ? (int)((key >> shift) & 255) : 256;
          const unsigned peers = __match_any_sync(0xffffffffu, d);
          const int rankW = __popc(peers & ((1u << lane) - 1u));
          const bool leader = lane == __ffs(peers) - 1;
          if (leader) wcnt[warp][d] = __popc(peers);
          __syncthreads();
          if (has) {
            int before = 0;
            for (int w = 0; w < warp; ++w) before += wcnt[w][d];
            const int dst = binStart[d] + run[d] + before + rankW;
            kd[s + dst] = key;
            id[s + dst] = val;
          }
          __syncthreads();
          if (leader && d < 256) atomicAdd(&run[d], __popc(peers));
          if (leader) wcnt[warp][d] = 0;
          __syncthreads();
        }
      }
    }
    // children: the left part keeps the first leftCount positions
    if (t == 0) {
      const uint32_t c = atomicAdd(A.taskCount, 2u);
      A.tasks[c] = Task{s, leftCount, T.obj, 0};
      A.tasks[c + 1] = Task{s + leftCount, count - leftCount, T.obj, 0};
      A.out[tid].left = (int32_t)c;
      A.out[tid].right = (int32_t)(c + 1);
    }
    __syncthreads();
  }
}

struct Buf {
  void *p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t bytes) { return cudaMalloc(&p, bytes ? bytes : 16); }
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

}  // namespace

extern "C" nomad_status nomad_scenebvh_build_gpu(const nomad_scene_desc *desc, int32_t device,
                                                 nomad_scenebvh **out) {
  if (!out) return NOMAD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  nomad_status st = nomad::scenebvh_validate(desc);
  if (st != NOMAD_OK) return st;
  NomadDeviceScope scope(device);  // outlives the device buffers below
  if (scope.err != cudaSuccess) {
    cudaGetLastError();
    return NOMAD_ERR_CUDA;
  }
  const uint32_t n = desc->prim_count, nobj = desc->object_count;
  try {
    std::vector<Task> level0;
    std::vector<int32_t> rootTask(nobj, -1);
    for (uint32_t o = 0; o < nobj; ++o)
      if (desc->object_prims[o] > 0) {
        rootTask[o] = (int32_t)level0.size();
        level0.push_back(Task{(int32_t)desc->object_first[o], (int32_t)desc->object_prims[o], (int32_t)o, 0});
      }
    const size_t cap = 2ull * n + nobj + 2;
    Buf dType, dGeom, dInfo, dIdx, dTmp, dKA, dKB, dTasks, dOut, dCount;
    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    if (!ok(dType.alloc((size_t)n * 4)) || !ok(dGeom.alloc((size_t)n * NOMAD_PRIM_GEOM_FLOATS * 4)) ||
        !ok(dInfo.alloc((size_t)n * 36)) || !ok(dIdx.alloc((size_t)n * 4)) || !ok(dTmp.alloc((size_t)n * 4)) ||
        !ok(dKA.alloc((size_t)n * 4)) || !ok(dKB.alloc((size_t)n * 4)) || !ok(dTasks.alloc(cap * sizeof(Task))) ||
        !ok(dOut.alloc(cap * sizeof(TaskOut))) || !ok(dCount.alloc(4))) {
      cudaGetLastError();
      return NOMAD_ERR_OUT_OF_MEMORY;
    }
    std::vector<int32_t> iota(n);
    for (uint32_t i = 0; i < n; ++i) iota[i] = (int32_t)i;
    const uint32_t n0 = (uint32_t)level0.size();
    bool good = ok(cudaMemcpy(dType.p, desc->prim_type, (size_t)n * 4, cudaMemcpyHostToDevice)) &&
                ok(cudaMemcpy(dGeom.p, desc->prim_geom, (size_t)n * NOMAD_PRIM_GEOM_FLOATS * 4,
                              cudaMemcpyHostToDevice)) &&
                ok(cudaMemcpy(dIdx.p, iota.data(), (size_t)n * 4, cudaMemcpyHostToDevice)) &&
                ok(cudaMemcpy(dTasks.p, level0.data(), n0 * sizeof(Task), cudaMemcpyHostToDevice)) &&
                ok(cudaMemcpy(dCount.p, &n0, 4, cudaMemcpyHostToDevice));
    if (!good) return NOMAD_ERR_CUDA;
    k_prim_info<<<(n + 255) / 256, 256>>>(dType.as<int32_t>(), dGeom.as<float>(), n, dInfo.as<float>());
    if (!ok(cudaGetLastError())) return NOMAD_ERR_CUDA;
    LevelArgs A{dInfo.as<float>(), dIdx.as<int32_t>(), dTmp.as<int32_t>(), dKA.as<uint32_t>(), dKB.as<uint32_t>(),
                dTasks.as<Task>(), dOut.as<TaskOut>(), dCount.as<uint32_t>(), 0, n0};
    uint32_t total = n0;
    while (A.lo < A.hi) {
      const uint32_t tasks = A.hi - A.lo;
      const unsigned grid = (unsigned)std::min<uint32_t>(tasks, 148u * 64u);
      k_build_level<<<grid, kB>>>(A);
      if (!ok(cudaGetLastError()) || !ok(cudaMemcpy(&total, dCount.p, 4, cudaMemcpyDeviceToHost)))
        return NOMAD_ERR_CUDA;
      if (total > cap) return NOMAD_ERR_LIMIT;
      A.lo = A.hi;
      A.hi = total;
    }
    std::vector<Task> tasks(total);
    std::vector<TaskOut> touts(total);
    std::vector<int32_t> idx(n);
    if (!ok(cudaMemcpy(tasks.data(), dTasks.p, total * sizeof(Task), cudaMemcpyDeviceToHost)) ||
        !ok(cudaMemcpy(touts.data(), dOut.p, total * sizeof(TaskOut), cudaMemcpyDeviceToHost)) ||
        !ok(cudaMemcpy(idx.data(), dIdx.p, (size_t)n * 4, cudaMemcpyDeviceToHost)))
      return NOMAD_ERR_CUDA;
    // pre-order numbering per object (node, left subtree, right subtree)
    std::vector<nomad::BlasResult> results(nobj);
    std::vector<int32_t> local(total, -1), order, stack;
    for (uint32_t o = 0; o < nobj; ++o) {
      if (rootTask[o] < 0) continue;
      order.clear();
      stack.assign(1, rootTask[o]);
      while (!stack.empty()) {
        const int32_t id = stack.back();
        stack.pop_back();
        local[id] = (int32_t)order.size();
        order.push_back(id);
        if (touts[id].left >= 0) {
          stack.push_back(touts[id].right);
          stack.push_back(touts[id].left);
        }
      }
      nomad::BlasResult &r = results[o];
      r.root = 0;
      r.nodes.resize(order.size());
      for (size_t k = 0; k < order.size(); ++k) {
        const TaskOut &to = touts[order[k]];
        nomad::BNode &b = r.nodes[k];
        b.mn = nomad::V3(to.mn[0], to.mn[1], to.mn[2]);
        b.mx = nomad::V3(to.mx[0], to.mx[1], to.mx[2]);
        if (to.left >= 0) {
          b.leftFirst = local[to.left];
          b.count = -local[to.right];
        } else {
          b.leftFirst = tasks[order[k]].start;
          b.count = tasks[order[k]].count;
        }
      }
    }
    std::unique_ptr<nomad_scenebvh> h(new nomad_scenebvh());
    st = nomad::scenebvh_finish(desc, results, idx, h->data, 0);
    if (st != NOMAD_OK) return st;
    *out = h.release();
    return NOMAD_OK;
  } catch (const std::bad_alloc &) {
    return NOMAD_ERR_OUT_OF_MEMORY;
  }
}
