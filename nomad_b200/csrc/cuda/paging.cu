// Geometry paging: per-object BLAS nodes and triangle records streamed between pinned host memory
// and a fixed device pool.
//
// The reference keeps one set of GPU resources per object (vertex/index buffers and a BLAS in a
// Metal heap) with the lifecycle Cold -> Streaming -> Resident (ResidentObjectGpuResources,
// Nomad Path Tracer/Renderer/Renderer.h:63-106; ensureResident, Renderer.cpp:613-650), starts at
// most kMaxColdObjectOnloadsPerFrame = 32 cold onloads per frame, denies onloads past the geometry
// cap and evicts objects that are no longer wanted (Renderer.cpp:5828-5905). Here the per-object
// resources are the object's nodes in one traversal layout and its triangle records:
//   * enable: every object's node block and record block (contiguous in the layouts) is copied
//     into a pinned "cold store" with refs made relative to the object (internal refs minus the
//     object's first node, leaf refs ~(record minus the object's first record)); the device arena
//     is replaced by [TLAS part of the layout][node pool][record pool], every instance link empty;
//   * onload: first-fit spans in the node and record pools, two cudaMemcpyAsync on a copy stream
//     (the copy engine) and a relocation kernel that adds the spans' bases to the refs, then an
//     event; the object stays Streaming (unlinked) until the event has completed, then its ref
//     is published: the ref table entry and, if the object is resident, its TLAS link;
//   * eviction: the link and the ref table entry are cleared at once on the compute stream; the
//     spans return to the free lists after an event recorded behind that clear (and behind the
//     object's copy, if it was still streaming) has completed, so no queued kernel reads reused
//     memory.
// Refs never leave the pools: a pool image only holds refs rebased into its own spans.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "rt_context.h"

using nomad::kEmptyRef;

namespace {

constexpr uint32_t kDefaultOnloads = 32;  // kMaxColdObjectOnloadsPerFrame (Renderer.cpp:5835)

// First-fit allocator over [0, cap) units, coalescing on release.
class RangeAlloc {
 public:
  void init(uint64_t cap) {
    free_.clear();
    if (cap) free_[0] = cap;
    used_ = 0;
  }
  bool alloc(uint64_t len, uint64_t &off) {
    if (len == 0) {
      off = 0;
      return true;
    }
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < len) continue;
      off = it->first;
      const uint64_t rest = it->second - len;
      free_.erase(it);
      if (rest) free_[off + len] = rest;
      used_ += len;
      return true;
    }
    return false;
  }
  void release(uint64_t off, uint64_t len) {
    if (len == 0) return;
    used_ -= len;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + len == next->first) {
      len += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += len;
        return;
      }
    }
    free_[off] = len;
  }
  uint64_t used() const { return used_; }

 private:
  std::map<uint64_t, uint64_t> free_;
  uint64_t used_ = 0;
};

struct Span {
  uint64_t off = 0, len = 0;
};

struct ObjPage {
  uint64_t imgNode = 0, nNodes = 0;  // node block in the cold store (node units)
  uint64_t imgRec = 0, nRecs = 0;    // record block in the cold store (record units)
  uint32_t firstRec = 0;             // leaf position of the object's first record
  int32_t rootRel = kEmptyRef;       // BLAS root ref relative to the object's blocks
  int64_t slotWord = -1;             // arena word of the object's TLAS link, -1 none
  Span node, rec;                    // pool spans while Streaming, Resident or Cached
  uint8_t state = NOMAD_PAGE_COLD;
  cudaEvent_t copied = nullptr;      // copy + relocation done
  int32_t poolRef = kEmptyRef;       // the relocated root ref of the pool copy
  uint64_t unwantedAt = 0;           // update count when it became Cached (LRU order)
};

struct Retire {
  Span node, rec;
  cudaEvent_t after = nullptr;  // compute-stream event behind the unlink (shared by one update's evictions)
  cudaEvent_t copy = nullptr;   // the object's copy event when it was still streaming (not owned)
  uint32_t obj = 0;
};

// One onload of a batch: where the object's blocks are in the cold store and in the pools.
struct StreamDesc {
  uint64_t imgNode, nNodes, imgRec, nRecs;
  int32_t nodeBase;  // absolute node index of the node span (TLAS part + pool offset)
  int32_t recBase;   // record pool index of the record span
  uint64_t dstNode;  // float4 offset of the node span in the arena
};

struct PubItem {
  uint32_t obj;
  int32_t ref;
};

struct Paging {
  uint32_t width = 0, fpn = 0;  // node layout width, floats per node
  uint32_t nodeBytes = 0;
  uint64_t tlasNodes = 0;       // the TLAS part kept at [0, tlasNodes)
  uint64_t nodeCap = 0, recCap = 0;
  uint64_t allNodes = 0, allRecs = 0;
  uint32_t maxOnloads = kDefaultOnloads;
  float *hostNodes = nullptr, *hostRecs = nullptr;  // pinned cold store
  const float4 *devNodes = nullptr, *devRecs = nullptr;  // the same, as the device maps it
  StreamDesc *pinnedDesc = nullptr;  // one update's onload batch
  DeviceBuf descBuf;
  cudaEvent_t descFree = nullptr;    // the previous batch's descriptors have been copied
  bool descPending = false;
  bool syncPublish = false;          // updates wait for the previous updates' copies and releases
  std::vector<ObjPage> obj;
  std::vector<int32_t> ref;     // host copy of the published ref table
  RangeAlloc nodeAlloc, recAlloc;
  std::vector<Retire> retiring;
  std::vector<cudaEvent_t> eventPool;  // unlink events not in use
  std::vector<uint32_t> recObject;  // leaf position -> object
  cudaStream_t copy = nullptr;
  cudaEvent_t lastCopy = nullptr;   // behind the latest copy queued
  bool anyCopy = false;
  PubItem *pinnedItems = nullptr;
  size_t pinnedCap = 0;
  cudaEvent_t itemsFree = nullptr;  // the previous publish copy has read the pinned items
  bool itemsPending = false;
  DeviceBuf items;
  DeviceBuf slots;  // arena word of each object's TLAS link (int64, -1 none)
  nomad_paging_stats stats{};
  uint64_t tick = 0;                // updates so far
  int32_t *refTable = nullptr;      // device ref table of the paged layout
  char *nodeBase = nullptr;         // arena: TLAS part then node pool
  float4 *recBase = nullptr;        // record pool
  ~Paging() {
    for (auto &o : obj)
      if (o.copied) cudaEventDestroy(o.copied);
    std::vector<cudaEvent_t> evs = eventPool;
    for (auto &r : retiring)
      if (r.after && std::find(evs.begin(), evs.end(), r.after) == evs.end()) evs.push_back(r.after);
    for (cudaEvent_t e : evs) cudaEventDestroy(e);
    if (lastCopy) cudaEventDestroy(lastCopy);
    if (itemsFree) cudaEventDestroy(itemsFree);
    if (copy) cudaStreamDestroy(copy);
    if (hostNodes) cudaFreeHost(hostNodes);
    if (hostRecs) cudaFreeHost(hostRecs);
    if (pinnedItems) cudaFreeHost(pinnedItems);
    if (pinnedDesc) cudaFreeHost(pinnedDesc);
    if (descFree) cudaEventDestroy(descFree);
  }
};

Paging *pg_of(const nomad_ctx *ctx) { return static_cast<Paging *>(ctx->paging); }

// Ref words of a node: pair nodes hold two refs (words 3 and 7), wide nodes W refs at 6W + k.
__device__ __forceinline__ uint32_t ref_word(uint32_t width, uint32_t k) {
  return width == 2 ? (k == 0 ? 3u : 7u) : 6u * width + k;
}

// Streams a batch of onloads in one launch, one block per object: the object's nodes and records
// are read from the pinned cold store (host memory the device maps) and written to their pool
// spans, the node refs rebased on the way (internal refs by the node span's absolute base, leaf
// refs ~record by the record span's base, empty refs unchanged).
__global__ void __launch_bounds__(256) k_stream_in(const StreamDesc *__restrict__ desc, const float4 *hostNodes,
                                                   const float4 *hostRecs, float4 *__restrict__ arena,
                                                   float4 *__restrict__ recPool, uint32_t fpn, uint32_t width) {
  const StreamDesc d = desc[blockIdx.x];
  const uint32_t q = fpn / 4;  // float4 per node
  const uint64_t nodeF4 = d.nNodes * q;
  for (uint64_t i = threadIdx.x; i < nodeF4; i += blockDim.x) {
    float4 v = hostNodes[d.imgNode * q + i];
    const uint32_t w0 = (uint32_t)(i % q) * 4;  // first word of this float4 within its node
    int32_t *w = reinterpret_cast<int32_t *>(&v);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const uint32_t word = w0 + (uint32_t)k;
      const bool isRef = width == 2 ? (word == 3 || word == 7) : (word >= 6 * width && word < 7 * width);
      if (!isRef) continue;
      const int32_t r = w[k];
      if (r >= 0)
        w[k] = r + d.nodeBase;
      else if (r != kEmptyRef)
        w[k] = ~((~r) + d.recBase);
    }
    arena[d.dstNode + i] = v;
  }
  const uint64_t recF4 = d.nRecs * 3;
  for (uint64_t i = threadIdx.x; i < recF4; i += blockDim.x)
    recPool[(uint64_t)d.recBase * 3 + i] = hostRecs[d.imgRec * 3 + i];
}

// Publishes refs: the ref table entry always, the TLAS link as the object's residency flag says
// (an empty ref clears the link).
__global__ void k_publish(const PubItem *__restrict__ items, uint32_t n, int32_t *__restrict__ refTable,
                          int32_t *__restrict__ arena, const long long *__restrict__ slotWord,
                          const uint8_t *__restrict__ res) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const PubItem it = items[i];
  refTable[it.obj] = it.ref;
  const long long w = slotWord[it.obj];
  if (w >= 0) arena[w] = (it.ref != kEmptyRef && res[it.obj]) ? it.ref : kEmptyRef;
}

nomad_status fail(nomad_ctx *ctx, nomad_status st, const std::string &m) { return nomad_fail(ctx, st, m); }

}  // namespace

void nomad_paging_free(nomad_ctx *ctx) {
  if (!ctx || !ctx->paging) return;
  Paging *pg = pg_of(ctx);
  if (pg->copy) cudaStreamSynchronize(pg->copy);
  delete pg;
  ctx->paging = nullptr;
  ctx->pagedWidth = 0;
}

int32_t nomad_paging_ref(const nomad_ctx *ctx, uint32_t obj) {
  const Paging *pg = pg_of(ctx);
  return pg && obj < pg->ref.size() ? pg->ref[obj] : kEmptyRef;
}

nomad_status nomad_paging_order(nomad_ctx *ctx) {
  Paging *pg = pg_of(ctx);
  if (!pg || !pg->anyCopy) return NOMAD_OK;
  NOMAD_CUDA(ctx, cudaEventRecord(pg->lastCopy, pg->copy));
  NOMAD_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, pg->lastCopy, 0));
  return NOMAD_OK;
}

int64_t nomad_paging_record_word(nomad_ctx *ctx, uint32_t pos, int32_t word) {
  Paging *pg = pg_of(ctx);
  if (!pg || pos >= pg->recObject.size()) return -1;
  const uint32_t o = pg->recObject[pos];
  ObjPage &op = pg->obj[o];
  const uint64_t local = pos - op.firstRec;
  int32_t *img = reinterpret_cast<int32_t *>(pg->hostRecs + (op.imgRec + local) * 12);
  img[3] = word;  // future onloads carry the new activity
  if (op.state == NOMAD_PAGE_COLD) return -1;
  const uint64_t recWord0 = (uint64_t)(reinterpret_cast<char *>(pg->recBase) - static_cast<char *>(ctx->arena.p)) / 4;
  return (int64_t)(recWord0 + (op.rec.off + local) * 12 + 3);
}

extern "C" nomad_status nomad_paging_enable(nomad_ctx *ctx, const nomad_paging_config *cfg) {
  if (!ctx || !cfg) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!ctx->sceneReady) return fail(ctx, NOMAD_ERR_NOT_READY, "no scene uploaded");
  if (ctx->paging) return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "paging is already enabled");
  if (cfg->width != 2 && cfg->width != 4 && cfg->width != 8)
    return fail(ctx, NOMAD_ERR_INVALID_ARGUMENT, "paged width must be 2, 4 or 8");
  NOMAD_DEVICE_SCOPE(ctx);
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  const nomad::TraversalLayout &L = ctx->layout;
  const uint32_t W = cfg->width, nobj = ctx->objectCount;
  const int wi = W == 4 ? 0 : 1;
  const nomad::WideLayout *WL = W == 2 ? nullptr : &ctx->wide[wi];
  const float *nodes = W == 2 ? L.pnodes.data() : WL->nodes.data();
  const uint32_t fpn = W == 2 ? 16u : WL->floatsPerNode;
  const uint64_t totalNodes = (W == 2 ? L.pnodes.size() : WL->nodes.size()) / fpn;
  const uint64_t tlas = W == 2 ? L.tlasPairCount : WL->tlasNodes;
  if (tlas == 0) return fail(ctx, NOMAD_ERR_UNSUPPORTED, "paging needs a TLAS with internal nodes");
  const uint32_t nref = W == 2 ? 2u : W;
  auto refw = [&](uint32_t k) { return W == 2 ? (k == 0 ? 3u : 7u) : 6u * W + k; };
  auto node_ref = [&](uint64_t n, uint32_t k) {
    int32_t r;
    std::memcpy(&r, nodes + n * fpn + refw(k), 4);
    return r;
  };

  std::unique_ptr<Paging> pg(new Paging());
  pg->width = W;
  pg->fpn = fpn;
  pg->nodeBytes = fpn * 4;
  pg->tlasNodes = tlas;
  pg->maxOnloads = cfg->max_onloads_per_frame ? cfg->max_onloads_per_frame : kDefaultOnloads;
  pg->obj.resize(nobj);
  pg->ref.assign(nobj, kEmptyRef);
  pg->recObject.assign(ctx->primCount, 0);
  // Per object: its node block (a DFS from the BLAS root must find a contiguous range after the
  // TLAS part) and its record block (the leaf positions of its primitives).
  std::vector<uint64_t> stack;
  for (uint32_t o = 0; o < nobj; ++o) {
    ObjPage &op = pg->obj[o];
    const nomad_instance_record &ir = ctx->instances[o];
    if (ir.primitive_count > 0) {
      uint32_t lo = UINT32_MAX, hi = 0;
      for (uint32_t p = ir.primitive_base; p < ir.primitive_base + ir.primitive_count; ++p) {
        const uint32_t pos = (uint32_t)L.primPos[p];
        lo = std::min(lo, pos);
        hi = std::max(hi, pos);
      }
      if (hi - lo + 1 != ir.primitive_count)
        return fail(ctx, NOMAD_ERR_UNSUPPORTED, "object " + std::to_string(o) + " records are not contiguous");
      op.firstRec = lo;
      op.nRecs = ir.primitive_count;
      for (uint32_t pos = lo; pos <= hi; ++pos) pg->recObject[pos] = o;
    }
    const int32_t root = W == 2 ? L.objBlasRef[o] : WL->objBlasRef[o];
    uint64_t nlo = UINT64_MAX, nhi = 0, count = 0;
    if (root >= 0) {
      stack.assign(1, (uint64_t)root);
      while (!stack.empty()) {
        const uint64_t n = stack.back();
        stack.pop_back();
        if (n >= totalNodes || n < tlas)
          return fail(ctx, NOMAD_ERR_UNSUPPORTED, "object " + std::to_string(o) + " nodes outside the BLAS part");
        ++count;
        nlo = std::min(nlo, n);
        nhi = std::max(nhi, n);
        for (uint32_t k = 0; k < nref; ++k) {
          const int32_t r = node_ref(n, k);
          if (r >= 0) stack.push_back((uint64_t)r);
        }
      }
      if (nhi - nlo + 1 != count)
        return fail(ctx, NOMAD_ERR_UNSUPPORTED, "object " + std::to_string(o) + " nodes are not contiguous");
      op.nNodes = count;
    }
    op.imgNode = pg->allNodes;
    op.imgRec = pg->allRecs;
    pg->allNodes += op.nNodes;
    pg->allRecs += op.nRecs;
    // relative root
    if (root >= 0)
      op.rootRel = (int32_t)((uint64_t)root - nlo);
    else if (root != kEmptyRef)
      op.rootRel = ~((~root) - (int32_t)op.firstRec);
    op.node.off = nlo;  // the object's first node, kept only until the image is filled below
  }
  // Cold store: node blocks with relative refs, record blocks verbatim.
  NOMAD_CUDA(ctx, cudaHostAlloc(&pg->hostNodes, std::max<uint64_t>(pg->allNodes, 1) * fpn * 4, cudaHostAllocMapped));
  NOMAD_CUDA(ctx, cudaHostAlloc(&pg->hostRecs, std::max<uint64_t>(pg->allRecs, 1) * 48, cudaHostAllocMapped));
  {
    void *dn = nullptr, *dr = nullptr;
    NOMAD_CUDA(ctx, cudaHostGetDevicePointer(&dn, pg->hostNodes, 0));
    NOMAD_CUDA(ctx, cudaHostGetDevicePointer(&dr, pg->hostRecs, 0));
    pg->devNodes = static_cast<const float4 *>(dn);
    pg->devRecs = static_cast<const float4 *>(dr);
  }
  NOMAD_CUDA(ctx, cudaHostAlloc(&pg->pinnedDesc, std::max<size_t>(nobj, 1) * sizeof(StreamDesc), cudaHostAllocDefault));
  NOMAD_CUDA(ctx, pg->descBuf.reserve(std::max<size_t>(nobj, 1) * sizeof(StreamDesc)));
  for (uint32_t o = 0; o < nobj; ++o) {
    ObjPage &op = pg->obj[o];
    const uint64_t nlo = op.node.off;
    op.node = Span{};
    if (op.nNodes) {
      float *dst = pg->hostNodes + op.imgNode * fpn;
      std::memcpy(dst, nodes + nlo * fpn, op.nNodes * fpn * 4);
      for (uint64_t i = 0; i < op.nNodes; ++i)
        for (uint32_t k = 0; k < nref; ++k) {
          int32_t r;
          std::memcpy(&r, dst + i * fpn + refw(k), 4);
          if (r >= 0) {
            r = (int32_t)((uint64_t)r - nlo);
          } else if (r != kEmptyRef) {
            const int64_t f = (int64_t)(~r) - op.firstRec;
            if (f < 0 || (uint64_t)f >= op.nRecs)
              return fail(ctx, NOMAD_ERR_UNSUPPORTED, "object " + std::to_string(o) + " leaf outside its records");
            r = ~(int32_t)f;
          }
          std::memcpy(dst + i * fpn + refw(k), &r, 4);
        }
    }
    if (op.nRecs)
      std::memcpy(pg->hostRecs + op.imgRec * 12, L.tris.data() + (uint64_t)op.firstRec * 12, op.nRecs * 48);
  }
  // Pool capacities: pool_bytes split in proportion to the scene's node and record bytes, never
  // more than the whole scene needs.
  const double nb = (double)pg->allNodes * pg->nodeBytes, rb = (double)pg->allRecs * 48.0;
  const double share = nb + rb > 0 ? nb / (nb + rb) : 0.5;
  pg->nodeCap = std::min<uint64_t>(pg->allNodes, (uint64_t)((double)cfg->pool_bytes * share) / pg->nodeBytes);
  pg->recCap = std::min<uint64_t>(pg->allRecs, (uint64_t)((double)cfg->pool_bytes * (1.0 - share)) / 48);
  if (pg->tlasNodes + pg->nodeCap > 0x7fffff00ull || pg->recCap > 0x7fffff00ull)
    return fail(ctx, NOMAD_ERR_LIMIT, "pool too large for 32-bit refs");
  pg->nodeAlloc.init(pg->nodeCap);
  pg->recAlloc.init(pg->recCap);
  // The TLAS part with every instance link empty.
  std::vector<float> tlasPart(nodes, nodes + tlas * fpn);
  const std::vector<int64_t> &slots = W == 2 ? L.objSlot : WL->objSlot;
  std::vector<long long> slotWord(nobj, -1);
  for (uint32_t o = 0; o < nobj; ++o) {
    const int64_t s = slots[o];
    if (s < 0) continue;
    const uint64_t node = W == 2 ? (uint64_t)s / 2 : (uint64_t)s / W;
    const uint32_t k = W == 2 ? (uint32_t)(s % 2) : (uint32_t)(s % W);
    if (node >= tlas) return fail(ctx, NOMAD_ERR_UNSUPPORTED, "instance link outside the TLAS part");
    const int32_t e = kEmptyRef;
    std::memcpy(tlasPart.data() + node * fpn + refw(k), &e, 4);
    slotWord[o] = (long long)(node * fpn + refw(k));
    pg->obj[o].slotWord = slotWord[o];
  }
  // New arena: [TLAS part][node pool][record pool].
  const size_t nodeRegion = (size_t)(tlas + pg->nodeCap) * pg->nodeBytes;
  DeviceBuf arena;
  NOMAD_CUDA(ctx, arena.reserve(nodeRegion + (size_t)pg->recCap * 48 + 256));
  NOMAD_CUDA(ctx, cudaMemset(arena.p, 0, arena.bytes));
  NOMAD_CUDA(ctx, cudaMemcpy(arena.p, tlasPart.data(), tlasPart.size() * 4, cudaMemcpyHostToDevice));
  NOMAD_CUDA(ctx, cudaStreamCreateWithFlags(&pg->copy, cudaStreamNonBlocking));
  NOMAD_CUDA(ctx, cudaEventCreateWithFlags(&pg->lastCopy, cudaEventDisableTiming));
  NOMAD_CUDA(ctx, cudaEventCreateWithFlags(&pg->itemsFree, cudaEventDisableTiming));
  NOMAD_CUDA(ctx, cudaEventCreateWithFlags(&pg->descFree, cudaEventDisableTiming));
  NOMAD_CUDA(ctx, cudaHostAlloc(&pg->pinnedItems, std::max<size_t>(nobj, 1) * sizeof(PubItem), cudaHostAllocDefault));
  pg->pinnedCap = std::max<size_t>(nobj, 1);
  NOMAD_CUDA(ctx, pg->items.reserve(pg->pinnedCap * sizeof(PubItem)));
  // Slot words and the ref table of the paged layout; the other layouts go away.
  ctx->frame.clearGraphs();
  ctx->arena.swap(arena);
  pg->nodeBase = static_cast<char *>(ctx->arena.p);
  pg->recBase = reinterpret_cast<float4 *>(pg->nodeBase + nodeRegion);
  nomad_ctx::Residency &R = ctx->res;
  std::vector<int32_t> empty(nobj, kEmptyRef);
  std::vector<long long> noSlot(nobj, -2);
  if (W == 2) {
    NOMAD_CUDA(ctx, cudaMemcpy(R.objBlasRef.p, empty.data(), (size_t)nobj * 4, cudaMemcpyHostToDevice));
    pg->refTable = R.objBlasRef.as<int32_t>();
    ctx->scene.pn = reinterpret_cast<const float4 *>(pg->nodeBase);
  } else {
    NOMAD_CUDA(ctx, cudaMemcpy(ctx->wideRef[wi].p, empty.data(), (size_t)nobj * 4, cudaMemcpyHostToDevice));
    NOMAD_CUDA(ctx, cudaMemcpy(R.objSlot.p, noSlot.data(), (size_t)nobj * 8, cudaMemcpyHostToDevice));
    pg->refTable = ctx->wideRef[wi].as<int32_t>();
    ctx->scene.pn = nullptr;
    ctx->ws[wi].wn = reinterpret_cast<const float4 *>(pg->nodeBase);
    ctx->wideWordBase[wi] = 0;
  }
  for (int w = 0; w < 2; ++w)
    if (W == 2 || w != wi) ctx->ws[w].wn = nullptr;
  ctx->scene.tri = pg->recBase;
  ctx->pnodeWords = nodeRegion / 4;
  // slot words on the device (for k_publish)
  NOMAD_CUDA(ctx, pg->slots.reserve((size_t)nobj * 8 + 8));
  NOMAD_CUDA(ctx, cudaMemcpy(pg->slots.p, slotWord.data(), (size_t)nobj * 8, cudaMemcpyHostToDevice));
  pg->stats.pool_bytes = pg->nodeCap * pg->nodeBytes + pg->recCap * 48;
  pg->stats.full_bytes = pg->allNodes * pg->nodeBytes + pg->allRecs * 48;
  pg->stats.cold = nobj;
  ctx->pagedWidth = W;
  ctx->paging = pg.release();
  if (!nomad_traversal_ok(ctx, ctx->trav, nullptr)) {
    nomad_traversal t = ctx->trav;
    t.width = W;
    t.persistent = 1;
    t.short_stack = t.staged_nodes = t.postpone_leaves = t.min_blocks = 0;
    t.regroup = 1;
    ctx->trav = t;
  }
  return NOMAD_OK;
}

namespace {

nomad_status publish(nomad_ctx *ctx, Paging *pg, const std::vector<PubItem> &items) {
  if (items.empty()) return NOMAD_OK;
  if (pg->itemsPending) NOMAD_CUDA(ctx, cudaEventSynchronize(pg->itemsFree));
  std::memcpy(pg->pinnedItems, items.data(), items.size() * sizeof(PubItem));
  NOMAD_CUDA(ctx, cudaMemcpyAsync(pg->items.p, pg->pinnedItems, items.size() * sizeof(PubItem),
                                  cudaMemcpyHostToDevice, ctx->stream));
  NOMAD_CUDA(ctx, cudaEventRecord(pg->itemsFree, ctx->stream));
  pg->itemsPending = true;
  const uint32_t n = (uint32_t)items.size();
  k_publish<<<(n + 255) / 256, 256, 0, ctx->stream>>>(pg->items.as<const PubItem>(), n, pg->refTable,
                                                      static_cast<int32_t *>(ctx->arena.p),
                                                      pg->slots.as<const long long>(),
                                                      ctx->res.objRes.as<const uint8_t>());
  NOMAD_CUDA(ctx, cudaGetLastError());
  return NOMAD_OK;
}

// Publishes every Streaming object whose copy has completed (or all of them, after a wait); one
// no longer wanted goes to the cache instead.
void collect_ready(const nomad_ctx *ctx, Paging *pg, std::vector<PubItem> &items, bool all) {
  for (uint32_t o = 0; o < pg->obj.size(); ++o) {
    ObjPage &op = pg->obj[o];
    if (op.state != NOMAD_PAGE_STREAMING) continue;
    if (!all && cudaEventQuery(op.copied) != cudaSuccess) continue;
    int32_t ref = op.rootRel;
    if (ref >= 0)
      ref = (int32_t)(pg->tlasNodes + op.node.off + (uint64_t)ref);
    else if (ref != kEmptyRef)
      ref = ~((~ref) + (int32_t)op.rec.off);
    op.poolRef = ref;
    --pg->stats.streaming;
    if (ctx->objResident[o]) {
      op.state = NOMAD_PAGE_RESIDENT;
      pg->ref[o] = ref;
      items.push_back(PubItem{o, ref});
      ++pg->stats.resident;
    } else {
      op.state = NOMAD_PAGE_CACHED;
      op.unwantedAt = pg->tick;
      ++pg->stats.cached;
    }
  }
}

void refresh_retired(Paging *pg) {
  size_t k = 0;
  std::vector<cudaEvent_t> done, busy;
  for (size_t i = 0; i < pg->retiring.size(); ++i) {
    Retire &r = pg->retiring[i];
    const bool ready = cudaEventQuery(r.after) == cudaSuccess && (!r.copy || cudaEventQuery(r.copy) == cudaSuccess);
    if (ready) {
      pg->nodeAlloc.release(r.node.off, r.node.len);
      pg->recAlloc.release(r.rec.off, r.rec.len);
      done.push_back(r.after);
    } else {
      busy.push_back(r.after);
      pg->retiring[k++] = r;
    }
  }
  pg->retiring.resize(k);
  // an unlink event returns to the pool once no pending retire shares it
  std::sort(done.begin(), done.end());
  done.erase(std::unique(done.begin(), done.end()), done.end());
  for (cudaEvent_t e : done)
    if (std::find(busy.begin(), busy.end(), e) == busy.end()) pg->eventPool.push_back(e);
}

}  // namespace

extern "C" nomad_status nomad_paging_update(nomad_ctx *ctx) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  Paging *pg = pg_of(ctx);
  if (!pg) return fail(ctx, NOMAD_ERR_NOT_READY, "paging is not enabled");
  NOMAD_DEVICE_SCOPE(ctx);
  nomad_status hs = nomad_residency_sync_host(ctx);
  if (hs != NOMAD_OK) return hs;
  if (pg->syncPublish) {
    // everything started or released by earlier updates completes before this one looks at it
    for (const ObjPage &op : pg->obj)
      if (op.state == NOMAD_PAGE_STREAMING) NOMAD_CUDA(ctx, cudaEventSynchronize(op.copied));
    for (const Retire &r : pg->retiring) {
      NOMAD_CUDA(ctx, cudaEventSynchronize(r.after));
      if (r.copy) NOMAD_CUDA(ctx, cudaEventSynchronize(r.copy));
    }
  }
  refresh_retired(pg);
  ++pg->tick;
  std::vector<PubItem> items;
  // Unwanted Resident objects are unlinked into the cache; wanted Cached ones relinked. Every
  // object gets at most one item per update.
  for (uint32_t o = 0; o < pg->obj.size(); ++o) {
    ObjPage &op = pg->obj[o];
    const bool want = ctx->objResident[o] != 0;
    if (!want && op.state == NOMAD_PAGE_RESIDENT) {
      op.state = NOMAD_PAGE_CACHED;
      op.unwantedAt = pg->tick;
      pg->ref[o] = kEmptyRef;
      items.push_back(PubItem{o, kEmptyRef});
      --pg->stats.resident;
      ++pg->stats.cached;
    } else if (want && op.state == NOMAD_PAGE_CACHED) {
      op.state = NOMAD_PAGE_RESIDENT;
      pg->ref[o] = op.poolRef;
      items.push_back(PubItem{o, op.poolRef});
      --pg->stats.cached;
      ++pg->stats.resident;
      ++pg->stats.relinks;
    }
  }
  collect_ready(ctx, pg, items, false);
  nomad_status st = publish(ctx, pg, items);
  if (st != NOMAD_OK) return st;
  // Releases cached copies, least recently unwanted first, until `nodes` and `recs` more units
  // are on their way back to the free lists (usable from a later update, once the work queued
  // before their unlink is done).
  uint64_t pendNodes = 0, pendRecs = 0;
  std::vector<Retire> retire;
  auto release_cache = [&](uint64_t nodes, uint64_t recs) {
    while (pendNodes < nodes || pendRecs < recs) {
      int64_t victim = -1;
      for (uint32_t o = 0; o < pg->obj.size(); ++o)
        if (pg->obj[o].state == NOMAD_PAGE_CACHED &&
            (victim < 0 || pg->obj[o].unwantedAt < pg->obj[victim].unwantedAt))
          victim = o;
      if (victim < 0) return false;
      ObjPage &vp = pg->obj[victim];
      retire.push_back(Retire{vp.node, vp.rec, nullptr, nullptr, (uint32_t)victim});
      pendNodes += vp.node.len;
      pendRecs += vp.rec.len;
      vp.state = NOMAD_PAGE_COLD;
      vp.node = vp.rec = Span{};
      vp.poolRef = kEmptyRef;
      --pg->stats.cached;
      ++pg->stats.cold;
      ++pg->stats.evictions;
    }
    return true;
  };
  // onloads, in object order, at most maxOnloads, streamed in by one launch on the copy stream
  uint32_t started = 0;
  std::vector<StreamDesc> batch;
  std::vector<uint32_t> batchObjs;
  for (uint32_t o = 0; o < pg->obj.size(); ++o) {
    ObjPage &op = pg->obj[o];
    if (!ctx->objResident[o] || op.state != NOMAD_PAGE_COLD || (op.nNodes == 0 && op.nRecs == 0)) continue;
    if (started >= pg->maxOnloads) {
      ++pg->stats.deferred;
      continue;
    }
    uint64_t noff = 0, roff = 0;
    bool got = pg->nodeAlloc.alloc(op.nNodes, noff);
    if (got && !pg->recAlloc.alloc(op.nRecs, roff)) {
      pg->nodeAlloc.release(noff, op.nNodes);
      got = false;
    }
    if (!got) {
      // make room from the cache for a later update; denied when the cache cannot
      if (!release_cache(pendNodes + op.nNodes, pendRecs + op.nRecs)) ++pg->stats.denied;
      else ++pg->stats.deferred;
      continue;
    }
    op.node = Span{noff, op.nNodes};
    op.rec = Span{roff, op.nRecs};
    if (!op.copied) NOMAD_CUDA(ctx, cudaEventCreateWithFlags(&op.copied, cudaEventDisableTiming));
    batch.push_back(StreamDesc{op.imgNode, op.nNodes, op.imgRec, op.nRecs, (int32_t)(pg->tlasNodes + noff),
                               (int32_t)roff, (pg->tlasNodes + noff) * (pg->fpn / 4)});
    batchObjs.push_back(o);
    op.state = NOMAD_PAGE_STREAMING;
    --pg->stats.cold;
    ++pg->stats.streaming;
    ++pg->stats.onloads;
    pg->stats.bytes_streamed += op.nNodes * pg->nodeBytes + op.nRecs * 48;
    ++started;
  }
  if (!batch.empty()) {
    if (pg->descPending) NOMAD_CUDA(ctx, cudaEventSynchronize(pg->descFree));
    std::memcpy(pg->pinnedDesc, batch.data(), batch.size() * sizeof(StreamDesc));
    NOMAD_CUDA(ctx, cudaMemcpyAsync(pg->descBuf.p, pg->pinnedDesc, batch.size() * sizeof(StreamDesc),
                                    cudaMemcpyHostToDevice, pg->copy));
    NOMAD_CUDA(ctx, cudaEventRecord(pg->descFree, pg->copy));
    pg->descPending = true;
    k_stream_in<<<(unsigned)batch.size(), 256, 0, pg->copy>>>(
        pg->descBuf.as<const StreamDesc>(), pg->devNodes, pg->devRecs, reinterpret_cast<float4 *>(pg->nodeBase),
        pg->recBase, pg->fpn, pg->width);
    NOMAD_CUDA(ctx, cudaGetLastError());
    for (uint32_t o : batchObjs) NOMAD_CUDA(ctx, cudaEventRecord(pg->obj[o].copied, pg->copy));
    pg->anyCopy = true;
  }
  if (!retire.empty()) {
    cudaEvent_t ev;
    if (!pg->eventPool.empty()) {
      ev = pg->eventPool.back();
      pg->eventPool.pop_back();
    } else {
      NOMAD_CUDA(ctx, cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    }
    NOMAD_CUDA(ctx, cudaEventRecord(ev, ctx->stream));
    for (Retire &r : retire) {
      r.after = ev;
      pg->retiring.push_back(r);
    }
  }
  return NOMAD_OK;
}

extern "C" nomad_status nomad_paging_wait(nomad_ctx *ctx) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  Paging *pg = pg_of(ctx);
  if (!pg) return fail(ctx, NOMAD_ERR_NOT_READY, "paging is not enabled");
  NOMAD_DEVICE_SCOPE(ctx);
  NOMAD_CUDA(ctx, cudaStreamSynchronize(pg->copy));
  std::vector<PubItem> items;
  collect_ready(ctx, pg, items, true);
  nomad_status st = publish(ctx, pg, items);
  if (st != NOMAD_OK) return st;
  NOMAD_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  refresh_retired(pg);
  return NOMAD_OK;
}

extern "C" nomad_status nomad_paging_set_sync(nomad_ctx *ctx, int32_t on) {
  if (!ctx) return NOMAD_ERR_INVALID_ARGUMENT;
  Paging *pg = pg_of(ctx);
  if (!pg) return fail(ctx, NOMAD_ERR_NOT_READY, "paging is not enabled");
  pg->syncPublish = on != 0;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_paging_stats_get(nomad_ctx *ctx, nomad_paging_stats *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  Paging *pg = pg_of(ctx);
  if (!pg) return fail(ctx, NOMAD_ERR_NOT_READY, "paging is not enabled");
  *out = pg->stats;
  out->used_bytes = pg->nodeAlloc.used() * pg->nodeBytes + pg->recAlloc.used() * 48;
  return NOMAD_OK;
}

extern "C" nomad_status nomad_paging_states(nomad_ctx *ctx, uint8_t *out) {
  if (!ctx || !out) return NOMAD_ERR_INVALID_ARGUMENT;
  Paging *pg = pg_of(ctx);
  if (!pg) return fail(ctx, NOMAD_ERR_NOT_READY, "paging is not enabled");
  for (size_t o = 0; o < pg->obj.size(); ++o) out[o] = pg->obj[o].state;
  return NOMAD_OK;
}
