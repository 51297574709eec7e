// libnomad_rt: CUDA context, scene upload, residency and the trace entry points of nomad_rt.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "rt_context.h"

using namespace nomad_dev;

namespace {

constexpr int kStack = 64;          // entries; the upload rejects deeper trees
constexpr int kBlock = 128;
constexpr int kPersistBlock = 128;

__device__ __forceinline__ void warp_count_object_hit(int32_t inst, uint32_t *counts) {
  unsigned mask = __activemask();
  unsigned peers = __match_any_sync(mask, inst);
  int lane = threadIdx.x & 31;
  int leader = __ffs(peers) - 1;
  if (inst >= 0 && lane == leader) atomicAdd(counts + inst, (uint32_t)__popc(peers));
}

__device__ __forceinline__ void store_hit(nomad_hit *out, uint64_t i, const HitRec &h) {
  int32_t *o = reinterpret_cast<int32_t *>(out + i);
  o[0] = h.inst;
  o[1] = h.prim;
  o[2] = __float_as_int(h.t);
  o[3] = __float_as_int(h.u);
  o[4] = __float_as_int(h.v);
}

// One kernel template for every traversal variant: width W (2 = pair nodes, 4, 8), stack size,
// closest or any hit, one ray per thread or persistent warps. Closest hits are written as
// (instance, primitive, t, u, v) words; lenDev, when set, holds the ray count on the device
// (ray queues of the path tracer).
template <int W, int STACK, bool ANY>
__device__ __forceinline__ void trace_one(const DevScene &S, const WideScene &WS, const RayP &r, float tmax,
                                          HitRec &h) {
  if (W == 2) {
    Work w{0, 0, 0};
    traverse<STACK, ANY, false>(S, r, tmax, h, w);
  } else {
    traverse_wide<W, STACK, ANY>(S, WS, r, tmax, h);
  }
}

template <int W, int STACK, bool ANY>
__device__ __forceinline__ void trace_ray(const DevScene &S, const WideScene &WS, const float4 *__restrict__ rays,
                                          uint64_t i, int32_t *__restrict__ hits5, uint8_t *__restrict__ occ,
                                          uint32_t *__restrict__ counts) {
  float4 a = __ldg(rays + 2 * i), b = __ldg(rays + 2 * i + 1);
  RayP r = prep_ray(a, b);
  HitRec h;
  trace_one<W, STACK, ANY>(S, WS, r, b.w, h);
  if (ANY) {
    occ[i] = h.prim >= 0 ? 1 : 0;
  } else {
    int32_t *o = hits5 + 5 * i;
    o[0] = h.inst;
    o[1] = h.prim;
    o[2] = __float_as_int(h.prim >= 0 ? h.t : INFINITY);
    o[3] = __float_as_int(h.u);
    o[4] = __float_as_int(h.v);
    if (counts) warp_count_object_hit(h.prim >= 0 ? h.inst : -1, counts);
  }
}

template <int W, int STACK, bool ANY, bool PERSIST, int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_trace(DevScene S, WideScene WS, const float4 *__restrict__ rays,
                                                  uint64_t n, const uint32_t *__restrict__ lenDev,
                                                  unsigned long long *__restrict__ cursor,
                                                  int32_t *__restrict__ hits5, uint8_t *__restrict__ occ,
                                                  uint32_t *__restrict__ counts) {
  const uint64_t N = lenDev ? (uint64_t)*lenDev : n;
  if (!PERSIST) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < N) trace_ray<W, STACK, ANY>(S, WS, rays, i, hits5, occ, counts);
    return;
  }
  int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(cursor, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= N) break;
    uint64_t i = base + lane;
    if (i < N) trace_ray<W, STACK, ANY>(S, WS, rays, i, hits5, occ, counts);
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kBlock) k_work(DevScene S, const float4 *__restrict__ rays,
                                                  uint64_t n, uint4 *__restrict__ out) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 a = __ldg(rays + 2 * i), b = __ldg(rays + 2 * i + 1);
  RayP r = prep_ray(a, b);
  HitRec h;
  Work w{0, 0, 0};
  traverse<kStack, false, true>(S, r, b.w, h, w);
  out[i] = make_uint4(w.nodes, w.tests, w.insts, h.prim >= 0 ? 1u : 0u);
}

// "Rays tested" per object: the resident objects whose TLAS leaf box (SceneBVH TLAS array:
// leaf left = -(object + 1)) the ray segment [1e-4, t of its closest hit] enters, infinite for a
// miss. A node's box contains its children's, and the slab test is monotone under containment,
// so walking the TLAS and pruning failed boxes finds exactly the leaves whose own box passes:
// the count does not depend on any traversal order. Each thread walks its rays in a grid-stride
// loop.
constexpr int kTlasStack = 64;

__global__ void __launch_bounds__(kBlock) k_object_tests(const float4 *__restrict__ tlas, const float4 *__restrict__ rays,
                                                         const int32_t *__restrict__ hits5, uint64_t n,
                                                         const uint32_t *__restrict__ lenDev,
                                                         const uint8_t *__restrict__ resident, uint32_t objects,
                                                         uint32_t *__restrict__ tests, uint32_t *__restrict__ status) {
  // Counts go to a per-block histogram in shared memory when it fits (one bin per object), and the
  // block adds its non-zero bins to the global counts once at the end: a ray enters a handful of
  // object boxes, and the popular objects would otherwise serialise on global atomics.
  extern __shared__ uint32_t hist[];
  const bool local = objects > 0;
  if (local) {
    for (uint32_t o = threadIdx.x; o < objects; o += blockDim.x) hist[o] = 0;
    __syncthreads();
  }
  const uint64_t N = lenDev ? (uint64_t)*lenDev : n;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += stride) {
    const float4 a = __ldg(rays + 2 * i), b = __ldg(rays + 2 * i + 1);
    const RayP r = prep_ray(a, b);
    const float bound = __int_as_float(hits5[5 * i + 2]);
    int32_t stack[kTlasStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
      const int32_t node = stack[--sp];
      const float4 lo = __ldg(tlas + 2 * node), hi = __ldg(tlas + 2 * node + 1);
      float tn;
      if (!slab(r, lo.x, lo.y, lo.z, hi.x, hi.y, hi.z, bound, tn)) continue;
      const int32_t left = __float_as_int(lo.w), right = __float_as_int(hi.w);
      if (left < 0) {
        const int32_t obj = -(left + 1);
        if (resident[obj]) {
          if (local)
            atomicAdd(&hist[obj], 1u);
          else
            atomicAdd(&tests[obj], 1u);
        }
        continue;
      }
      if (sp + 2 > kTlasStack) {
        atomicOr(status, kStatusStackOverflow);
        continue;
      }
      stack[sp++] = right;
      stack[sp++] = left;
    }
  }
  if (local) {
    __syncthreads();
    for (uint32_t o = threadIdx.x; o < objects; o += blockDim.x)
      if (hist[o]) atomicAdd(tests + o, hist[o]);
  }
}

// Instance slots of the wide layouts from the device residency flags.
__global__ void k_patch_wide(int32_t *__restrict__ arena, size_t base, uint32_t fpn, uint32_t width,
                             const long long *__restrict__ slot, const int32_t *__restrict__ ref,
                             const uint8_t *__restrict__ res, uint32_t n) {
  uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  long long s = slot[o];
  if (s < 0) return;
  arena[base + (size_t)(s / width) * fpn + 6 * width + (size_t)(s % width)] = res[o] ? ref[o] : kEmptyRef;
}

// Residency patches: word offsets into the layout arena and their new values.
// Device primitive-activity flags from a list of changed primitives: bit 31 the new state, bits
// 0-30 the primitive.
__global__ void k_set_prim_act(uint8_t *__restrict__ act, const uint32_t *__restrict__ list, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) act[list[i] & 0x7fffffffu] = (uint8_t)(list[i] >> 31);
}

__global__ void k_patch(int32_t *__restrict__ arena, const int64_t *__restrict__ offs,
                        const int32_t *__restrict__ vals, uint32_t n) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) arena[offs[i]] = vals[i];
}

}  // namespace

namespace {

nomad_status fail(nomad_ctx *c, nomad_status st, const std::string &msg) {
  return nomad_fail(c, st, msg);
}

bool is_device_ptr(const void *p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

}  // namespace

extern "C" nomad_status nomad_create(const nomad_config *cfg, nomad_ctx **out) {
  if (!out) return NOMAD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  const int device = cfg ? cfg->device : 0;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) {
    cudaGetLastError();
    return NOMAD_ERR_CUDA;
  }
  if (device < 0 || device >= count) return NOMAD_ERR_INVALID_ARGUMENT;
  NomadDeviceScope scope(device);  // outlives the context's buffers on every failure path
  if (scope.err != cudaSuccess) return NOMAD_ERR_CUDA;
  std::unique_ptr<nomad_ctx> c(new (std::nothrow) nomad_ctx());
  if (!c) return NOMAD_ERR_OUT_OF_MEMORY;
  c->device = device;
  if (nomad_noalloc_lookup(device) != cudaSuccess) return NOMAD_ERR_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, c->device) != cudaSuccess) return NOMAD_ERR_CUDA;
  if (prop.major < 10) return NOMAD_ERR_UNSUPPORTED;  // built for sm_100a only
  c->smCount = prop.multiProcessorCount;
  if (nomad_regroup_init() != cudaSuccess) return NOMAD_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&c->ownStream, cudaStreamNonBlocking) != cudaSuccess)
    return NOMAD_ERR_CUDA;
  c->stream = c->ownStream;
  for (auto &s : c->copyStreams)
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return NOMAD_ERR_CUDA;
  if (c->status.reserve(16) != cudaSuccess || c->cursor.reserve(64) != cudaSuccess)
    return NOMAD_ERR_OUT_OF_MEMORY;
  cudaMemset(c->status.p, 0, 16);
  *out = c.release();
  return NOMAD_OK;
}

extern "C" nomad_status nomad_destroy(nomad_ctx *ctx) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  {
    NomadDeviceScope scope(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    for (auto s : ctx->copyStreams)
      if (s) cudaStreamDestroy(s);
    if (ctx->ownStream) cudaStreamDestroy(ctx->ownStream);
    if (ctx->mlp) nomad_mlp_free(ctx->mlp);
    nomad_paging_free(ctx);
    delete ctx;  // frees the context's device buffers with its device current
  }
  return NOMAD_OK;
}

extern "C" const char *nomad_last_error(const nomad_ctx *ctx) {
  return ctx ? ctx->err.c_str() : "null context";
}

extern "C" nomad_status nomad_sync(nomad_ctx *ctx) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_set_stream(nomad_ctx *ctx, void *cuda_stream) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  ctx->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : ctx->ownStream;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_get_status(nomad_ctx *ctx, uint32_t *word) {
  if (!ctx || !word) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(word, ctx->status.p, 4, cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaMemsetAsync(ctx->status.p, 0, 4, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_scene_upload(nomad_ctx *ctx, const float *bvh, uint32_t bvhCount,
                                           const float *tlas, uint32_t tlasCount,
                                           const float *prims, const float *materials,
                                           const int32_t *primIndices, uint32_t primCount,
                                           const nomad_instance_record *inst,
                                           uint32_t objectCount) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!bvh || !tlas || !prims || !materials || !primIndices || !inst)
    return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "null scene array");
  NOMAD_DEVICE_SCOPE(ctx);
  if (ctx->resHostStale) {  // a pending flag copy must land before the pinned buffer is reused
    NOMAD_CUDA(ctx, cudaEventSynchronize(ctx->resEvent));
    ctx->resHostStale = false;
  }
  ctx->sceneReady = false;
  if (ctx->paging) {  // a new scene ends paging: the arena is rebuilt whole below
    nomad_paging_free(ctx);
    ctx->frame.clearGraphs();
  }
  // Leaf refs are ~first record; the values just above INT32_MIN are kernel sentinels.
  if (primCount > 0x7ffffff0u) return fail(ctx, NOMAD_ERR_LIMIT, "too many primitives");
  std::vector<nomad::ObjectRange> objs(objectCount);
  for (uint32_t o = 0; o < objectCount; ++o)
    objs[o] = {inst[o].blas_root_index, inst[o].primitive_base, inst[o].primitive_count};
  std::string err;
  try {
    if (!nomad::build_traversal_layout(bvh, bvhCount, tlas, tlasCount, prims, primIndices,
                                       primCount, objs.data(), objectCount, ctx->layout,
                                       ctx->objResident, err))
      return fail(ctx, NOMAD_ERR_SCENE_INVALID, err);
  } catch (const std::bad_alloc &) {
    return fail(ctx, NOMAD_ERR_OUT_OF_MEMORY, "host memory");
  }
  if (ctx->layout.maxDepth > (uint32_t)kStack)
    return fail(ctx, NOMAD_ERR_LIMIT,
                "tree depth " + std::to_string(ctx->layout.maxDepth) + " exceeds the traversal stack");
  const auto &L = ctx->layout;
  ctx->stackNeed[0] = L.maxDepth;
  try {
    for (int w = 0; w < 2; ++w) {
      nomad::build_wide_layout(L, w == 0 ? 4 : 8, ctx->objResident, ctx->wide[w]);
      ctx->stackNeed[1 + w] = (ctx->wide[w].width - 1) * ctx->wide[w].maxDepth;
    }
  } catch (const std::bad_alloc &) {
    return fail(ctx, NOMAD_ERR_OUT_OF_MEMORY, "host memory");
  }
  size_t pnBytes = L.pnodes.size() * 4, triBytes = L.tris.size() * 4;
  size_t wBytes[2] = {ctx->wide[0].nodes.size() * 4, ctx->wide[1].nodes.size() * 4};
  NOMAD_CUDA(ctx, ctx->arena.reserve(pnBytes + triBytes + wBytes[0] + wBytes[1] + 256));
  NOMAD_CUDA(ctx, ctx->prims.reserve((size_t)primCount * 112));
  NOMAD_CUDA(ctx, ctx->materials.reserve((size_t)primCount * 80));
  NOMAD_CUDA(ctx, ctx->objHits.reserve((size_t)objectCount * 4 + 16));
  char *base = static_cast<char *>(ctx->arena.p);
  if (pnBytes)
    NOMAD_CUDA(ctx, cudaMemcpy(base, L.pnodes.data(), pnBytes, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(base + pnBytes, L.tris.data(), triBytes, cudaMemcpyHostToDevice));
  {
    size_t off = pnBytes + triBytes;
    for (int w = 0; w < 2; ++w) {
      const nomad::WideLayout &WL = ctx->wide[w];
      if (wBytes[w]) NOMAD_CUDA(ctx, cudaMemcpy(base + off, WL.nodes.data(), wBytes[w], cudaMemcpyHostToDevice));
      ctx->wideWordBase[w] = off / 4;
      ctx->ws[w].wn = reinterpret_cast<const float4 *>(base + off);
      ctx->ws[w].root = WL.rootRef;
      NOMAD_CUDA(ctx, ctx->wideSlot[w].reserve((size_t)objectCount * 8 + 8));
      NOMAD_CUDA(ctx, ctx->wideRef[w].reserve((size_t)objectCount * 4 + 4));
      NOMAD_CUDA(ctx, cudaMemcpy(ctx->wideSlot[w].p, WL.objSlot.data(), (size_t)objectCount * 8, cudaMemcpyHostToDevice));
      NOMAD_CUDA(ctx, cudaMemcpy(ctx->wideRef[w].p, WL.objBlasRef.data(), (size_t)objectCount * 4, cudaMemcpyHostToDevice));
      off += wBytes[w];
    }
  }
  NOMAD_CUDA(ctx, cudaMemcpy(ctx->prims.p, prims, (size_t)primCount * 112, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemcpy(ctx->materials.p, materials, (size_t)primCount * 80,
                             cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaMemset(ctx->objHits.p, 0, (size_t)objectCount * 4 + 16));
  {
    nomad_status ss = nomad_build_shade_records(ctx, materials, primCount);
    if (ss != NOMAD_OK) return ss;
  }
  ctx->pnodeWords = pnBytes / 4;
  DevScene &S = ctx->scene;
  S.pn = reinterpret_cast<const float4 *>(base);
  S.tri = reinterpret_cast<const float4 *>(base + pnBytes);
  S.prims = static_cast<const float4 *>(ctx->prims.p);
  for (int k = 0; k < 3; ++k) {
    S.rmin[k] = L.rootMin[k];
    S.rmax[k] = L.rootMax[k];
  }
  S.rootRef = L.rootRef;
  S.tlasPairs = L.tlasPairCount;
  S.status = static_cast<uint32_t *>(ctx->status.p);
  ctx->primCount = primCount;
  ctx->objectCount = objectCount;
  ctx->primActive.assign(primCount, 1);
  ctx->objActiveCount.assign(objectCount, 0);
  for (uint32_t o = 0; o < objectCount; ++o) ctx->objActiveCount[o] = inst[o].primitive_count;
  ctx->instances.assign(inst, inst + objectCount);
  ctx->hostPrims.assign(prims, prims + (size_t)primCount * 28);
  ctx->res.hostTlas.assign(tlas, tlas + (size_t)tlasCount * 8);
  ctx->res.tlasCount = tlasCount;
  ctx->hostMaterials.assign(materials, materials + (size_t)primCount * 20);
  ctx->frame.lightsDirty = true;
  ctx->frame.restirValid = false;
  ctx->res.bvhNodeCount = bvhCount;
  ctx->dirtyPrims.clear();
  ctx->dirtyObjs.clear();
  ctx->primDirtyFlag.assign(primCount, 0);
  ctx->objDirtyFlag.assign(objectCount, 0);
  // Objects uploaded non-resident keep their primitives flagged active (like the reference,
  // where residency is per object through the instance record); they are skipped via the TLAS.
  nomad_status rst = nomad_residency_init(ctx);
  if (rst != NOMAD_OK) return rst;
  ctx->sceneReady = true;
  // A configuration chosen for another scene may need a deeper stack or more nodes than this one has.
  if (!nomad_traversal_ok(ctx, ctx->trav, nullptr)) ctx->trav = nomad_kernel_config(NOMAD_KERNEL_BVH2);
  return NOMAD_OK;
}

namespace {
// setPrimitiveActive's bookkeeping for one primitive (the host mirror is current, the index valid);
// returns whether its state changed.
bool toggle_primitive(nomad_ctx *ctx, uint32_t prim, uint8_t a) {
  if (ctx->primActive[prim] == a) return false;
  ctx->primActive[prim] = a;
  uint32_t o = static_cast<uint32_t>(ctx->layout.primObject[prim]);
  if (a)
    ++ctx->objActiveCount[o];
  else if (ctx->objActiveCount[o] > 0)
    --ctx->objActiveCount[o];
  if (!ctx->primDirtyFlag[prim]) {
    ctx->primDirtyFlag[prim] = 1;
    ctx->dirtyPrims.push_back(prim);
  }
  if (!ctx->objDirtyFlag[o]) {
    ctx->objDirtyFlag[o] = 1;
    ctx->dirtyObjs.push_back(o);
  }
  return true;
}
}  // namespace

extern "C" nomad_status nomad_residency_set_primitive_active(nomad_ctx *ctx, uint32_t prim,
                                                             int32_t active, int32_t *changed) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  {
    nomad_status hs = nomad_residency_sync_host(ctx);
    if (hs != NOMAD_OK) return hs;
  }
  if (changed) *changed = 0;
  if (prim >= ctx->primCount) return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "primitive out of range");
  if (!toggle_primitive(ctx, prim, active ? 1 : 0)) return NOMAD_OK;
  if (changed) *changed = 1;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_set_object_active(nomad_ctx *ctx, uint32_t obj,
                                                          int32_t active, uint32_t *toggled) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  {
    nomad_status hs = nomad_residency_sync_host(ctx);
    if (hs != NOMAD_OK) return hs;
  }
  if (toggled) *toggled = 0;
  if (obj >= ctx->objectCount) return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "object out of range");
  const nomad_instance_record &r = ctx->instances[obj];
  uint32_t n = 0;
  for (uint32_t p = r.primitive_base; p < r.primitive_base + r.primitive_count; ++p)
    n += toggle_primitive(ctx, p, active ? 1 : 0) ? 1u : 0u;
  // An object toggled with no primitive change still gets its instance record refreshed.
  if (!ctx->objDirtyFlag[obj]) {
    ctx->objDirtyFlag[obj] = 1;
    ctx->dirtyObjs.push_back(obj);
  }
  if (toggled) *toggled = n;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_flush(nomad_ctx *ctx) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  {
    nomad_status hs = nomad_residency_sync_host(ctx);
    if (hs != NOMAD_OK) return hs;
  }
  std::vector<int64_t> offs;
  std::vector<int32_t> vals;
  const auto &L = ctx->layout;
  if (ctx->paging) {  // patches below must land after the copies that may hold these records
    nomad_status ps = nomad_paging_order(ctx);
    if (ps != NOMAD_OK) return ps;
  }
  std::vector<uint32_t> primList;  // changed primitives for the device activity flags
  primList.reserve(ctx->dirtyPrims.size());
  for (uint32_t p : ctx->dirtyPrims) {
    ctx->primDirtyFlag[p] = 0;
    primList.push_back(p | (ctx->primActive[p] ? 0x80000000u : 0u));
    int64_t pos = L.primPos[p];
    const int32_t word = ctx->primActive[p] ? (int32_t)p : ~(int32_t)p;
    if (ctx->paging) {
      const int64_t w = nomad_paging_record_word(ctx, (uint32_t)pos, word);
      if (w < 0) continue;  // a Cold object: its host copy holds the new word
      offs.push_back(w);
    } else {
      offs.push_back((int64_t)ctx->pnodeWords + pos * 12 + 3);
    }
    vals.push_back(word);
  }
  for (uint32_t o : ctx->dirtyObjs) {
    ctx->objDirtyFlag[o] = 0;
    bool res = ctx->objActiveCount[o] > 0 && ctx->instances[o].primitive_count > 0;
    ctx->objResident[o] = res ? 1 : 0;
    int32_t ref = res ? (ctx->paging ? nomad_paging_ref(ctx, o) : L.objBlasRef[o]) : nomad::kEmptyRef;
    // Instance record as the reference fills it (Renderer.cpp:5344-5357).
    ctx->instances[o].blas_root_index = res ? L.objRootNode[o] : -1;
    // pair-layout links exist unless a wide layout is paged
    int64_t slot = (ctx->pagedWidth == 0 || ctx->pagedWidth == 2) ? L.objSlot[o] : -2;
    if (slot == -1) {
      ctx->scene.rootRef = ref;
    } else if (slot >= 0) {
      int64_t pair = slot / 2, side = slot % 2;
      offs.push_back(pair * 16 + (side == 0 ? 3 : 7));
      vals.push_back(ref);
    }
  }
  bool mirror = !ctx->dirtyPrims.empty() || !ctx->dirtyObjs.empty();
  ctx->dirtyPrims.clear();
  ctx->dirtyObjs.clear();
  if (mirror) {
    nomad_status mst;
    if ((uint64_t)primList.size() * 16 < ctx->primCount) {
      // few changes: the object flags whole, the primitive flags by a scatter of the changed ones
      // (a full copy moves one byte per primitive of the scene)
      auto &R = ctx->res;
      NOMAD_CUDA(ctx, cudaMemcpyAsync(R.objRes.p, ctx->objResident.data(), ctx->objectCount, cudaMemcpyHostToDevice,
                                      ctx->stream));
      if (!primList.empty()) {
        NOMAD_CUDA(ctx, ctx->patchPrims.reserve(primList.size() * 4));
        NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->patchPrims.p, primList.data(), primList.size() * 4,
                                        cudaMemcpyHostToDevice, ctx->stream));
        const uint32_t n = (uint32_t)primList.size();
        k_set_prim_act<<<(n + 255) / 256, 256, 0, ctx->stream>>>(R.primAct.as<uint8_t>(),
                                                                 ctx->patchPrims.as<const uint32_t>(), n);
        NOMAD_CUDA(ctx, cudaGetLastError());
      }
      ctx->frame.lightsDirty = true;
      mst = NOMAD_OK;
    } else {
      mst = nomad_residency_mirror(ctx);
    }
    if (mst != NOMAD_OK) return mst;
    mst = nomad_patch_wide(ctx);
    if (mst != NOMAD_OK) return mst;
  }
  if (offs.empty()) {
    NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));  // primList leaves scope
    return NOMAD_OK;
  }
  NOMAD_CUDA(ctx, ctx->patchOffs.reserve(offs.size() * 8));
  NOMAD_CUDA(ctx, ctx->patchVals.reserve(vals.size() * 4));
  // Synchronous copies: the host vectors go out of scope at return.
  NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->patchOffs.p, offs.data(), offs.size() * 8,
                                  cudaMemcpyHostToDevice, ctx->stream));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->patchVals.p, vals.data(), vals.size() * 4,
                                  cudaMemcpyHostToDevice, ctx->stream));
  uint32_t n = static_cast<uint32_t>(offs.size());
  k_patch<<<(n + 255) / 256, 256, 0, ctx->stream>>>(static_cast<int32_t *>(ctx->arena.p),
                                                    static_cast<const int64_t *>(ctx->patchOffs.p),
                                                    static_cast<const int32_t *>(ctx->patchVals.p), n);
  NOMAD_CUDA(ctx, cudaGetLastError());
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_residency_get_instances(nomad_ctx *ctx, nomad_instance_record *out) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  {
    nomad_status hs = nomad_residency_sync_host(ctx);
    if (hs != NOMAD_OK) return hs;
  }
  if (!out) return NOMAD_ERR_INVALID_ARGUMENT;
  for (uint32_t o = 0; o < ctx->objectCount; ++o) {
    out[o] = ctx->instances[o];
    if (!ctx->objResident[o]) out[o].blas_root_index = -1;
  }
  return NOMAD_OK;
}

namespace {

// Stack entries of each variant: pair nodes 64; 4-wide 64; 8-wide 96.
constexpr int kStackW4 = 64, kStackW8 = 96;

template <int W, int STACK, bool ANY, bool PERSIST, int MINB>
nomad_status launch_one(nomad_ctx *ctx, const WideScene &WS, const float4 *rays, uint64_t n, const uint32_t *lenDev,
                        unsigned long long *cursor, int32_t *hits5, uint8_t *occ, uint32_t *counts, cudaStream_t st) {
  auto kern = k_trace<W, STACK, ANY, PERSIST, MINB>;
  uint64_t blocks;
  if (PERSIST) {
    int perSm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kern, kBlock, 0);
    blocks = (uint64_t)ctx->smCount * std::max(perSm, 1);
    blocks = std::max<uint64_t>(1, std::min(blocks, (n + kBlock - 1) / kBlock));
    NOMAD_CUDA(ctx, cudaMemsetAsync(cursor, 0, 8, st));
  } else {
    blocks = (n + kBlock - 1) / kBlock;
    if (blocks > 0x7fffffffull) return nomad_fail(ctx, NOMAD_ERR_LIMIT, "too many rays for one call");
  }
  kern<<<(unsigned)blocks, kBlock, 0, st>>>(ctx->scene, WS, rays, n, lenDev, cursor, hits5, occ, counts);
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

template <int W, int STACK, bool ANY, bool PERSIST>
nomad_status launch_minb(nomad_ctx *ctx, uint32_t minBlocks, const WideScene &WS, const float4 *rays, uint64_t n,
                         const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5, uint8_t *occ,
                         uint32_t *counts, cudaStream_t st) {
  switch (minBlocks) {
    case 0: return launch_one<W, STACK, ANY, PERSIST, 1>(ctx, WS, rays, n, lenDev, cursor, hits5, occ, counts, st);
    case 10: return launch_one<W, STACK, ANY, PERSIST, 10>(ctx, WS, rays, n, lenDev, cursor, hits5, occ, counts, st);
    case 12: return launch_one<W, STACK, ANY, PERSIST, 12>(ctx, WS, rays, n, lenDev, cursor, hits5, occ, counts, st);
    case 16: return launch_one<W, STACK, ANY, PERSIST, 16>(ctx, WS, rays, n, lenDev, cursor, hits5, occ, counts, st);
    default: return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "min_blocks must be 0, 10, 12 or 16");
  }
}

template <bool ANY>
nomad_status dispatch(nomad_ctx *ctx, const nomad_traversal &c, const float4 *rays, uint64_t n, const uint32_t *lenDev,
                      unsigned long long *cursor, int32_t *hits5, uint8_t *occ, uint32_t *counts, cudaStream_t st) {
  const WideScene none{nullptr, kEmptyRef};
  const bool p = c.persistent != 0;
  const uint32_t mb = c.min_blocks;
  switch (c.width) {
    case 2: return p ? launch_minb<2, kStack, ANY, true>(ctx, mb, none, rays, n, lenDev, cursor, hits5, occ, counts, st)
                     : launch_minb<2, kStack, ANY, false>(ctx, mb, none, rays, n, lenDev, cursor, hits5, occ, counts, st);
    case 4: return p ? launch_minb<4, kStackW4, ANY, true>(ctx, mb, ctx->ws[0], rays, n, lenDev, cursor, hits5, occ, counts, st)
                     : launch_minb<4, kStackW4, ANY, false>(ctx, mb, ctx->ws[0], rays, n, lenDev, cursor, hits5, occ, counts, st);
    case 8: return p ? launch_minb<8, kStackW8, ANY, true>(ctx, mb, ctx->ws[1], rays, n, lenDev, cursor, hits5, occ, counts, st)
                     : launch_minb<8, kStackW8, ANY, false>(ctx, mb, ctx->ws[1], rays, n, lenDev, cursor, hits5, occ, counts, st);
    default: return nomad_fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "unknown kernel variant");
  }
}

}  // namespace

nomad_status nomad_trace_variant(nomad_ctx *ctx, const nomad_traversal &cfg, bool any, const float4 *rays, uint64_t n,
                                 const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5,
                                 uint8_t *occ, uint32_t *counts, cudaStream_t st) {
  if (n == 0) return NOMAD_OK;
  std::string why;
  if (!nomad_traversal_ok(ctx, cfg, &why)) return nomad_fail(ctx, NOMAD_ERR_UNSUPPORTED, why);
  if (cfg.persistent == 2)
    return nomad_trace_regroup(ctx, cfg, any, rays, n, lenDev, cursor, hits5, occ, counts, st);
  if (cfg.persistent == 3)
    return nomad_trace_packet(ctx, cfg, any, rays, n, lenDev, cursor, hits5, occ, counts, st);
  return any ? dispatch<true>(ctx, cfg, rays, n, lenDev, cursor, hits5, occ, counts, st)
             : dispatch<false>(ctx, cfg, rays, n, lenDev, cursor, hits5, occ, counts, st);
}

extern "C" nomad_status nomad_set_kernel(nomad_ctx *ctx, uint32_t kernel) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (kernel == NOMAD_KERNEL_AUTO) kernel = NOMAD_KERNEL_BVH2;
  if (kernel >= NOMAD_KERNEL_COUNT) return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "unknown kernel");
  const nomad_traversal c = nomad_kernel_config(kernel);
  if (ctx->sceneReady && !nomad_traversal_ok(ctx, c, nullptr))
    return fail(ctx, NOMAD_ERR_UNSUPPORTED, "kernel variant needs a deeper stack than it has for this scene");
  ctx->trav = c;
  return NOMAD_OK;
}

namespace {

// Launches one of the trace kernels over device arrays on `st`; `slot` picks the cursor word
// (one per stream that may run a persistent kernel concurrently).
enum class Op { Closest, Any, Work };

nomad_status launch(nomad_ctx *ctx, Op op, const float4 *rays, uint64_t n, void *out,
                    bool countHits, cudaStream_t st, int slot = 0) {
  if (n == 0) return NOMAD_OK;
  uint32_t *counts = countHits ? static_cast<uint32_t *>(ctx->objHits.p) : nullptr;
  unsigned long long *cursor = static_cast<unsigned long long *>(ctx->cursor.p) + slot;
  if (op == Op::Work) {
    uint64_t blocks = (n + kBlock - 1) / kBlock;
    if (blocks > 0x7fffffffull) return fail(ctx, NOMAD_ERR_LIMIT, "too many rays for one call");
    k_work<<<(unsigned)blocks, kBlock, 0, st>>>(ctx->scene, rays, n, static_cast<uint4 *>(out));
    NOMAD_CUDA(ctx, cudaGetLastError());
    return NOMAD_OK;
  }
  if (op == Op::Any)
    return nomad_trace_variant(ctx, ctx->trav, true, rays, n, nullptr, cursor, nullptr, static_cast<uint8_t *>(out),
                               nullptr, st);
  nomad_status rs = nomad_trace_variant(ctx, ctx->trav, false, rays, n, nullptr, cursor,
                                        static_cast<int32_t *>(out), nullptr, counts, st);
  if (rs != NOMAD_OK || !countHits) return rs;
  // st is the context's stream on every caller's path
  return nomad_count_object_tests(ctx, rays, static_cast<const int32_t *>(out), n, nullptr);
}

// Host-pointer path: rays are copied in and results out in chunks, alternating two streams
// so one chunk's copies overlap another chunk's traversal.
// Host buffers: the batch is split into chunks; uploads run back to back on one copy stream,
// each chunk's kernel on the context stream once its upload landed, and each chunk's download on
// a second copy stream once its kernel finished, so both copy directions and the traversal
// overlap.
nomad_status trace_host(nomad_ctx *ctx, Op op, const nomad_ray *rays, uint64_t n, void *out,
                        size_t outStride, bool countHits) {
  NOMAD_CUDA(ctx, ctx->stageIn.reserve(n * sizeof(nomad_ray)));
  NOMAD_CUDA(ctx, ctx->stageOut.reserve(n * outStride));
  // Chunks of a sixteenth of the batch (at least 2^19 rays). The last chunk's traversal and
  // download run after every upload has landed, so a batch of more than two chunks ends with
  // halving ones (1/2, 1/4, 1/8, 1/8 of a chunk): the part of the batch that no upload overlaps
  // shrinks to an eighth of a chunk.
  const uint64_t chunk = std::max<uint64_t>(1 << 19, (n + 15) / 16);
  std::vector<uint64_t> parts;
  {
    uint64_t rest = n;
    const bool taper = n > 2 * chunk;
    while (rest > (taper ? chunk : 0)) {
      const uint64_t m = std::min(chunk, rest);
      parts.push_back(m);
      rest -= m;
    }
    const uint64_t last = std::max<uint64_t>(chunk / 8, 1 << 16);
    while (rest > last) {
      const uint64_t m = (rest + 1) / 2;
      parts.push_back(m);
      rest -= m;
    }
    if (rest > 0) parts.push_back(rest);
  }
  cudaStream_t sIn = ctx->copyStreams[0], sOut = ctx->copyStreams[1], sK = ctx->stream;
  std::vector<cudaEvent_t> evs;
  auto event = [&](cudaEvent_t *e) -> cudaError_t {
    cudaError_t r = cudaEventCreateWithFlags(e, cudaEventDisableTiming);
    if (r == cudaSuccess) evs.push_back(*e);
    return r;
  };
  auto cleanup = [&]() {
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
  };
  nomad_status st = NOMAD_OK;
  cudaEvent_t start;
  if (event(&start) != cudaSuccess || cudaEventRecord(start, sK) != cudaSuccess ||
      cudaStreamWaitEvent(sIn, start, 0) != cudaSuccess)
    st = fail(ctx, NOMAD_ERR_CUDA, "stream setup");
  // Uploads and kernels first, downloads second: a copy to or from pageable host memory returns
  // only once it is done, so issuing a download before the next upload would serialise them.
  std::vector<cudaEvent_t> traced;
  uint64_t off = 0;
  for (size_t k = 0; k < parts.size() && st == NOMAD_OK; off += parts[k], ++k) {
    const uint64_t m = parts[k];
    char *din = static_cast<char *>(ctx->stageIn.p) + off * sizeof(nomad_ray);
    char *dout = static_cast<char *>(ctx->stageOut.p) + off * outStride;
    cudaEvent_t up, done;
    if (event(&up) != cudaSuccess || event(&done) != cudaSuccess ||
        cudaMemcpyAsync(din, rays + off, m * sizeof(nomad_ray), cudaMemcpyHostToDevice, sIn) != cudaSuccess ||
        cudaEventRecord(up, sIn) != cudaSuccess || cudaStreamWaitEvent(sK, up, 0) != cudaSuccess) {
      st = fail(ctx, NOMAD_ERR_CUDA, "chunk upload");
      break;
    }
    st = launch(ctx, op, reinterpret_cast<const float4 *>(din), m, dout, countHits, sK, 0);
    if (st != NOMAD_OK) break;
    if (cudaEventRecord(done, sK) != cudaSuccess) {
      st = fail(ctx, NOMAD_ERR_CUDA, "chunk event");
      break;
    }
    traced.push_back(done);
  }
  off = 0;
  for (size_t k = 0; k < traced.size() && st == NOMAD_OK; off += parts[k], ++k) {
    const uint64_t m = parts[k];
    if (cudaStreamWaitEvent(sOut, traced[k], 0) != cudaSuccess ||
        cudaMemcpyAsync(static_cast<char *>(out) + off * outStride,
                        static_cast<char *>(ctx->stageOut.p) + off * outStride, m * outStride,
                        cudaMemcpyDeviceToHost, sOut) != cudaSuccess)
      st = fail(ctx, NOMAD_ERR_CUDA, "chunk download");
  }
  // wait for every stream the batch touched, also after an error, before buffers are reused
  cudaError_t e1 = cudaStreamSynchronize(sIn), e2 = cudaStreamSynchronize(sK), e3 = cudaStreamSynchronize(sOut);
  cleanup();
  if (st != NOMAD_OK) return st;
  if (e1 != cudaSuccess) return nomad_cuda_fail(ctx, e1, "upload stream");
  if (e2 != cudaSuccess) return nomad_cuda_fail(ctx, e2, "trace stream");
  if (e3 != cudaSuccess) return nomad_cuda_fail(ctx, e3, "download stream");
  return NOMAD_OK;
}

nomad_status trace_entry(nomad_ctx *ctx, Op op, const nomad_ray *rays, uint64_t n, void *out,
                         size_t outStride, uint32_t flags) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady) return fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (n == 0) return NOMAD_OK;
  if (!rays || !out) return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "null rays or output");
  NOMAD_DEVICE_SCOPE(ctx);
  bool countHits = (flags & NOMAD_TRACE_COUNT_HITS) != 0 && op == Op::Closest;
  if (flags & NOMAD_TRACE_DEVICE_POINTERS) {
    if (reinterpret_cast<uintptr_t>(rays) % 16 != 0)
      return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "device rays must be 16-byte aligned");
    return launch(ctx, op, reinterpret_cast<const float4 *>(rays), n, out, countHits, ctx->stream);
  }
  if (is_device_ptr(rays) || is_device_ptr(out))
    return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT,
                "device pointer passed without NOMAD_TRACE_DEVICE_POINTERS");
  return trace_host(ctx, op, rays, n, out, outStride, countHits);
}

}  // namespace

extern "C" nomad_status nomad_trace_closest(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n,
                                            nomad_hit *out, uint32_t flags) {
  return trace_entry(ctx, Op::Closest, rays, n, out, sizeof(nomad_hit), flags);
}

extern "C" nomad_status nomad_trace_any(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n,
                                        uint8_t *out, uint32_t flags) {
  return trace_entry(ctx, Op::Any, rays, n, out, 1, flags);
}

extern "C" nomad_status nomad_trace_work(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n,
                                         uint32_t *out, uint32_t flags) {
  if (ctx && ctx->pagedWidth > 2)
    return fail(ctx, NOMAD_ERR_UNSUPPORTED, "the counting walk needs the pair layout, which is not on the device while a wide layout is paged");
  return trace_entry(ctx, Op::Work, rays, n, out, 16, flags);
}

extern "C" nomad_status nomad_read_object_hits(nomad_ctx *ctx, uint32_t *out) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  if (!out) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(out, ctx->objHits.p, (size_t)ctx->objectCount * 4,
                                  cudaMemcpyDeviceToHost, ctx->stream));
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_read_object_hits_ex(nomad_ctx *ctx, uint32_t *out, uint32_t flags) {
  if (!(flags & NOMAD_TRACE_DEVICE_POINTERS)) return nomad_read_object_hits(ctx, out);
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  if (!out) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  NOMAD_CUDA(ctx, cudaMemcpyAsync(out, ctx->objHits.p, (size_t)ctx->objectCount * 4, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_write_object_hits(nomad_ctx *ctx, const uint32_t *counts, uint32_t flags) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  if (!counts) return NOMAD_ERR_INVALID_ARGUMENT;
  NOMAD_DEVICE_SCOPE(ctx);
  const bool dev = (flags & NOMAD_TRACE_DEVICE_POINTERS) != 0;
  NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->objHits.p, counts, (size_t)ctx->objectCount * 4,
                                  dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, ctx->stream));
  // a host source may go out of scope when the call returns
  if (!dev) NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return NOMAD_OK;
}

extern "C" nomad_status nomad_reset_object_hits(nomad_ctx *ctx) {
  if (!ctx || !ctx->sceneReady) return NOMAD_ERR_NOT_READY;
  NOMAD_DEVICE_SCOPE(ctx);
  NOMAD_CUDA(ctx, cudaMemsetAsync(ctx->objHits.p, 0, (size_t)ctx->objectCount * 4, ctx->stream));
  return NOMAD_OK;
}

// ---------------------------------------------------------------------------------------------
// Allocation-free closest hit with per-object hit counts.
//
// For callers that cannot allocate GPU memory at trace time: a frame loop that has committed
// its whole geometry budget to resident objects (every byte is accounted by the residency
// manager), or one that cannot afford the implicit device synchronisation that cudaMalloc and
// cudaFree may cause in the middle of a frame. The persistent closest-hit kernel needs scratch
// memory (a work cursor and per-object hit accumulators); here that scratch is a fixed
// file-scope device array instead of memory allocated per context or per call.
//
// Limits and behaviour:
//   * at most kNoAllocMaxObjects objects (64 KiB of accumulators + one 256-byte cursor line);
//     larger scenes are rejected with NOMAD_ERR_LIMIT;
//   * the array lives in every GPU that loads this library, until the process exits;
//   * the array's device address is looked up (cudaGetSymbolAddress, with that device current)
//     when a context is created on a device, and by the first call on a device that has none
//     cached; make that first call before any stream capture. The lookup is repeated by every
//     nomad_create, so contexts created after a cudaDeviceReset use the reloaded module's array;
//   * every call shares the one array: calls on the same device that overlap on the GPU (two
//     streams, or two contexts) race on it. Serialise them;
//   * each call clears the cursor and the accumulators it uses before the launch.
namespace {

constexpr uint32_t kNoAllocMaxObjects = 16384;
constexpr uint32_t kNoAllocCursorWords = 64;  // one 256-byte line holding the 64-bit cursor
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocCursorWords + kNoAllocMaxObjects];

// Per device: the scratch array's device address (null until looked up). Atomic, so host threads
// that make their first call at the same time may both look it up and store the same address.
std::atomic<uint32_t *> g_noalloc_addr[kNoAllocMaxDevices] = {};

__global__ void __launch_bounds__(kPersistBlock) k_closest_persist_noalloc(
    DevScene S, const float4 *__restrict__ rays, uint64_t n, nomad_hit *__restrict__ out,
    uint32_t *__restrict__ scratch) {
  unsigned long long *cursor = reinterpret_cast<unsigned long long *>(scratch);
  uint32_t *counts = scratch + kNoAllocCursorWords;
  int lane = threadIdx.x & 31;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(cursor, 32ull);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= n) break;
    uint64_t i = base + lane;
    if (i < n) {
      float4 a = __ldg(rays + 2 * i), b = __ldg(rays + 2 * i + 1);
      RayP r = prep_ray(a, b);
      HitRec h;
      Work w{0, 0, 0};
      traverse<kStack, false, false>(S, r, b.w, h, w);
      if (h.prim < 0) h.t = INFINITY;
      store_hit(out, i, h);
      warp_count_object_hit(h.prim >= 0 ? h.inst : -1, counts);
    }
    __syncwarp();
  }
}

}  // namespace

cudaError_t nomad_noalloc_lookup(int device) {
  if (device < 0 || device >= kNoAllocMaxDevices) return cudaSuccess;  // the entry point refuses it
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return e;
  g_noalloc_addr[device].store(static_cast<uint32_t *>(p), std::memory_order_release);
  return cudaSuccess;
}

extern "C" nomad_status nomad_trace_closest_noalloc(nomad_ctx *ctx, const nomad_ray *d_rays,
                                                    uint64_t n, nomad_hit *d_hits,
                                                    uint32_t *d_object_hits) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady) return fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (ctx->pagedWidth > 2)
    return fail(ctx, NOMAD_ERR_UNSUPPORTED, "the allocation-free walk needs the pair layout, which is not on the device while a wide layout is paged");
  if (ctx->objectCount > kNoAllocMaxObjects)
    return fail(ctx, NOMAD_ERR_LIMIT,
                "nomad_trace_closest_noalloc supports at most " +
                    std::to_string(kNoAllocMaxObjects) + " objects; the scene has " +
                    std::to_string(ctx->objectCount));
  if (!d_rays || !d_hits || !d_object_hits)
    return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "null device pointer");
  if (reinterpret_cast<uintptr_t>(d_rays) % 16 != 0)
    return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "device rays must be 16-byte aligned");
  if (ctx->device < 0 || ctx->device >= kNoAllocMaxDevices)
    return fail(ctx, NOMAD_ERR_LIMIT, "device ordinal too large for the static scratch table");
  NOMAD_DEVICE_SCOPE(ctx);
  uint32_t *scratch = g_noalloc_addr[ctx->device].load(std::memory_order_acquire);
  if (!scratch) {
    NOMAD_CUDA(ctx, nomad_noalloc_lookup(ctx->device));
    scratch = g_noalloc_addr[ctx->device].load(std::memory_order_acquire);
  }
  size_t clearBytes = (kNoAllocCursorWords + (size_t)ctx->objectCount) * 4;
  NOMAD_CUDA(ctx, cudaMemsetAsync(scratch, 0, clearBytes, ctx->stream));
  if (n > 0) {
    int perSm = 0;
    NOMAD_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, k_closest_persist_noalloc,
                                                                  kPersistBlock, 0));
    perSm = std::max(perSm, 1);
    uint64_t blocks = (uint64_t)ctx->smCount * perSm;
    blocks = std::max<uint64_t>(1, std::min(blocks, (n + kPersistBlock - 1) / kPersistBlock));
    k_closest_persist_noalloc<<<(unsigned)blocks, kPersistBlock, 0, ctx->stream>>>(
        ctx->scene, reinterpret_cast<const float4 *>(d_rays), n, d_hits, scratch);
    NOMAD_CUDA(ctx, cudaGetLastError());
  }
  NOMAD_CUDA(ctx, cudaMemcpyAsync(d_object_hits, scratch + kNoAllocCursorWords,
                                  (size_t)ctx->objectCount * 4, cudaMemcpyDeviceToDevice,
                                  ctx->stream));
  return NOMAD_OK;
}

nomad_status nomad_count_object_tests(nomad_ctx *ctx, const float4 *rays, const int32_t *hits5, uint64_t n,
                                      const uint32_t *lenDev) {
  auto &R = ctx->res;
  if (!R.testsOn || n == 0 || R.tlasCount == 0) return NOMAD_OK;
  // a grid-stride launch of a few blocks per SM, each with a histogram of every object (at most
  // 16,384 objects: 64 KB of shared memory; larger scenes count straight into global memory)
  const uint32_t objects = ctx->objectCount <= 16384 ? ctx->objectCount : 0u;
  const size_t smem = (size_t)objects * 4;
  if (smem > 48 * 1024 && !ctx->objTestsSmemSet) {
    NOMAD_CUDA(ctx, cudaFuncSetAttribute(k_object_tests, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * 1024));
    ctx->objTestsSmemSet = true;
  }
  const uint64_t blocks = std::min<uint64_t>((n + kBlock - 1) / kBlock, (uint64_t)ctx->smCount * 8);
  k_object_tests<<<(unsigned)std::max<uint64_t>(blocks, 1), kBlock, smem, ctx->stream>>>(
      R.tlas.as<const float4>(), rays, hits5, n, lenDev, R.objRes.as<const uint8_t>(), objects,
      R.tests.as<uint32_t>(), ctx->status.as<uint32_t>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

nomad_status nomad_patch_wide(nomad_ctx *ctx) {
  const uint32_t n = ctx->objectCount;
  for (int w = 0; w < 2; ++w) {
    const nomad::WideLayout &WL = ctx->wide[w];
    if (!WL.width) continue;
    if (ctx->pagedWidth && ctx->pagedWidth != WL.width) continue;  // not on the device while paging
    k_patch_wide<<<(n + 255) / 256, 256, 0, ctx->stream>>>(static_cast<int32_t *>(ctx->arena.p), ctx->wideWordBase[w],
                                                          WL.floatsPerNode, WL.width, ctx->wideSlot[w].as<const long long>(),
                                                          ctx->wideRef[w].as<const int32_t>(),
                                                          ctx->res.objRes.as<const uint8_t>(), n);
    NOMAD_CUDA(ctx, cudaGetLastError());
    if (ctx->layout.tlasPairCount == 0)  // the single object is the root: its ref lives on the host
      for (uint32_t o = 0; o < n; ++o)
        if (WL.objSlot[o] == -1) ctx->ws[w].root = ctx->objResident[o] ? WL.objBlasRef[o] : kEmptyRef;
  }
  return NOMAD_OK;
}

extern "C" nomad_status nomad_autotune(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n, uint32_t repeats,
                                       uint32_t flags, nomad_tune_result *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady) return fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (!rays || n == 0) return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "no sample rays");
  NOMAD_DEVICE_SCOPE(ctx);
  cudaStream_t s = ctx->stream;
  const float4 *d = reinterpret_cast<const float4 *>(rays);
  if (!(flags & NOMAD_TRACE_DEVICE_POINTERS)) {
    NOMAD_CUDA(ctx, ctx->stageIn.reserve(n * sizeof(nomad_ray)));
    NOMAD_CUDA(ctx, cudaMemcpyAsync(ctx->stageIn.p, rays, n * sizeof(nomad_ray), cudaMemcpyHostToDevice, s));
    d = ctx->stageIn.as<const float4>();
  }
  DeviceBuf ref, cur;
  NOMAD_CUDA(ctx, ref.reserve(n * 20));
  NOMAD_CUDA(ctx, cur.reserve(n * 20));
  std::vector<int32_t> hRef(n * 5), hCur(n * 5);
  cudaEvent_t e0, e1;
  NOMAD_CUDA(ctx, cudaEventCreate(&e0));
  NOMAD_CUDA(ctx, cudaEventCreate(&e1));
  std::memset(out, 0, sizeof(*out));
  for (int w = 0; w < 3; ++w) out->stack_need[w] = ctx->stackNeed[w];
  float bestMs = 1e30f;
  uint32_t best = NOMAD_KERNEL_BVH2;
  unsigned long long *cursor = static_cast<unsigned long long *>(ctx->cursor.p);
  for (uint32_t k = NOMAD_KERNEL_BVH2; k < NOMAD_KERNEL_COUNT; ++k) {
    out->ms[k] = -1.0f;
    const nomad_traversal cfg = nomad_kernel_config(k);
    if (!nomad_traversal_ok(ctx, cfg, nullptr)) continue;
    DeviceBuf &dst = (k == NOMAD_KERNEL_BVH2) ? ref : cur;
    float t = 1e30f;
    for (uint32_t rep = 0; rep < std::max(1u, repeats) + 1; ++rep) {
      NOMAD_CUDA(ctx, cudaEventRecord(e0, s));
      nomad_status st = nomad_trace_variant(ctx, cfg, false, d, n, nullptr, cursor, dst.as<int32_t>(), nullptr, nullptr, s);
      if (st != NOMAD_OK) return st;
      NOMAD_CUDA(ctx, cudaEventRecord(e1, s));
      NOMAD_CUDA(ctx, cudaEventSynchronize(e1));
      float ms = 0.0f;
      NOMAD_CUDA(ctx, cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0) t = std::min(t, ms);  // first launch is a warm-up
    }
    out->ms[k] = t;
    if (k == NOMAD_KERNEL_BVH2) {
      NOMAD_CUDA(ctx, cudaMemcpy(hRef.data(), ref.p, n * 20, cudaMemcpyDeviceToHost));
    } else {
      NOMAD_CUDA(ctx, cudaMemcpy(hCur.data(), cur.p, n * 20, cudaMemcpyDeviceToHost));
      uint32_t bad = 0;
      for (uint64_t i = 0; i < n; ++i)
        if (std::memcmp(&hRef[5 * i], &hCur[5 * i], 20) != 0) ++bad;
      out->mismatches[k] = bad;
      if (bad) continue;  // a variant that disagrees is never chosen
    }
    if (t < bestMs) {
      bestMs = t;
      best = k;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx->trav = nomad_kernel_config(best);
  out->best = best;
  return NOMAD_OK;
}
