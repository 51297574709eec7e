// Internal: the libnomad_rt context shared by the traversal (rt_core.cu) and the path tracer
// (pathtrace.cu) translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <utility>
#include <vector>

#include "../../../include/nomad_rt.h"
#include "../host/layout.h"
#include "device_scope.h"
#include "rt_device.cuh"
#include "rt_wide.cuh"

struct DeviceBuf {
  void *p = nullptr;
  size_t bytes = 0;
  DeviceBuf() = default;
  DeviceBuf(const DeviceBuf &) = delete;
  DeviceBuf &operator=(const DeviceBuf &) = delete;
  ~DeviceBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t reserve(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <typename T> T *as() const { return static_cast<T *>(p); }
  void swap(DeviceBuf &o) {
    std::swap(p, o.p);
    std::swap(bytes, o.bytes);
  }
};

// Light tables on the device: rebuilt by one kernel whenever residency changes.
struct LightMeta {
  uint32_t count;
  float total;
};

// Device buffers of the wavefront path tracer (one slot per path; see pathtrace.cu).
struct FrameState {
  uint64_t capacity = 0;  // paths
  DeviceBuf thr, rad;                 // float4 per path
  DeviceBuf qRays[2], qIds[2];        // ray queues (2 float4 + id per entry)
  DeviceBuf hits;                     // 5 words per queue entry
  DeviceBuf sRays, sIds, sContrib;    // shadow queue
  DeviceBuf sOcc;                     // 1 byte per shadow entry
  DeviceBuf counters;                 // queue lengths, cursors, statistics
  DeviceBuf views;                    // view table
  DeviceBuf lightIdx, lightCdf, lightPdf, lightMeta;
  DeviceBuf lightRec;                 // per CDF slot, 5 float4 (pt_lights.cuh)
  bool lightsDirty = true;
  // ReSTIR DI: per-path reservoirs (initial, temporal, final of this and the previous frame),
  // surface records (this and the previous frame) and the previous frame's view table
  DeviceBuf rInit, rTemp, resv[2], surf[2], prevViews;
  uint64_t restirPaths = 0;
  int restirCur = 0;
  bool restirValid = false;
  nomad_restir_config restir{32, 1, 3, 30.0f, 20.0f, 0};
  // reference-mode ReSTIR: candidate and reuse visibility queues, per-path visibility masks,
  // the selected contribution after the candidates
  DeviceBuf refRays, refIds, refOcc, refMask, reuseMask, refContrib;
  uint64_t refRayCap = 0, refPaths = 0;
  std::vector<nomad_view> prevHostViews;
  // Captured frames: one CUDA graph per frame shape (sizes, buffers, traversal configuration,
  // scene parameters); the view table is read from device memory, so cameras, seeds and frame
  // numbers change without a new capture.
  struct Graph {
    std::vector<unsigned char> key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint64_t lastUse = 0;
  };
  std::vector<Graph> graphs;
  uint64_t graphTick = 0;
  uint64_t graphCaptures = 0, graphLaunches = 0;
  void clearGraphs() {
    for (Graph &g : graphs) {
      if (g.exec) cudaGraphExecDestroy(g.exec);
      if (g.graph) cudaGraphDestroy(g.graph);
    }
    graphs.clear();
  }
  ~FrameState() { clearGraphs(); }
};

struct nomad_ctx {
  int device = 0;
  int smCount = 0;
  cudaStream_t stream = nullptr;     // stream used by calls (own or caller's)
  cudaStream_t ownStream = nullptr;
  cudaStream_t copyStreams[2] = {nullptr, nullptr};
  std::string err;
  nomad_traversal trav{2, 0, 0, 1, 0, 128, 0, 0};  // kernel configuration of the trace calls
  bool sceneReady = false;
  // scene sizes
  uint32_t primCount = 0, objectCount = 0;
  // device memory
  DeviceBuf arena;      // pair nodes then triangle records
  DeviceBuf prims, materials;
  // Compact shading records: one float4 per primitive (the geometric-or-shading normal the hit
  // normal resolves to, or a sphere's center, and bits(material index | type << 30)) and the
  // distinct 80-byte material records they index (nomad_build_shade_records).
  DeviceBuf shadeRec, matTable;
  DeviceBuf patchPrims;          // changed primitives of a flush (k_set_prim_act)
  bool objTestsSmemSet = false;  // k_object_tests opted in to 64 KB of dynamic shared memory
  uint32_t matCount = 0;
  DeviceBuf objHits, status, cursor;
  DeviceBuf stageIn, stageOut, stageAux;  // host-pointer staging
  DeviceBuf patchOffs, patchVals;
  size_t pnodeWords = 0;  // int32 words of the pair-node part of the arena
  nomad_dev::DevScene scene{};
  // wide layouts (4 and 8 children) in the same arena
  nomad::WideLayout wide[2];
  size_t wideWordBase[2] = {0, 0};
  nomad_dev::WideScene ws[2] = {};
  uint32_t stackNeed[3] = {0, 0, 0};  // stack entries a walk can need: binary, 4-wide, 8-wide
  DeviceBuf wideSlot[2], wideRef[2];
  // host copies needed by the light tables
  std::vector<float> hostPrims, hostMaterials;
  // host residency state
  nomad::TraversalLayout layout;
  std::vector<uint8_t> primActive, objResident;
  std::vector<uint32_t> objActiveCount;
  std::vector<nomad_instance_record> instances;
  std::vector<uint32_t> dirtyPrims, dirtyObjs;
  std::vector<uint8_t> primDirtyFlag, objDirtyFlag;
  // path tracer
  FrameState frame;
  // device residency state (residency.cu)
  struct Residency {
    bool ready = false;
    uint32_t bvhNodeCount = 0;
    DeviceBuf objSlot, objBlasRef, objRes, primAct;   // int64, int32, u8, u8
    DeviceBuf bounds, bytes, tris, emit;               // float4 (centre, radius), u64, u32, f32
    DeviceBuf score, hist, lastHit, prevDist, visible; // f32, u32[8], u32, f32, u8
    DeviceBuf features, keys, desired, misc;           // f32[24], f32, u8, misc words
    DeviceBuf emissive;                                // {prim, weight bits, object} per emissive primitive
    uint32_t emissiveCount = 0;
    uint32_t frame = 0;
    float prevCam[3] = {0, 0, 0};
    bool havePrevCam = false;
    std::vector<uint64_t> hostBytes;
    // per-primitive ray-hit policy (NOMAD_POLICY_RAYHIT_PRIM): device hit counters (counted by the
    // path tracer once enabled) and the host-side state of the reference's policy
    bool primHitsOn = false;
    DeviceBuf primHits;
    std::vector<uint32_t> primHitsHost;
    // Per-primitive cooldowns of the per-primitive ray-hit and ScreenSpace policies, stored as the
    // step at which they run out: a primitive is cooling while primCooldown[p] > primStep, and
    // each step of either policy advances primStep instead of decrementing every counter.
    std::vector<uint32_t> primCooldown;
    uint32_t primStep = 0;
    std::vector<float> primScore;
    std::vector<float> primSphere;  // centre xyz, radius per primitive
    std::vector<uint8_t> primVisible;
    uint32_t primRebuild = 0;
    // learned-policy steps that ran the ray-hit budget for want of a usable model
    uint64_t fallbackSteps = 0;
    // Per-object Beta hit-probability posterior (processRayHitCounters, Renderer.cpp:8004-8522),
    // fed by per-object closest hits and "rays tested": the closest-hit ray segments that enter
    // the object's TLAS leaf box before their hit (counted on the device once testsOn is set).
    // post: per object alpha, beta, probability, variance, mass, exploration (f32) then idle
    // frames, hits and tests of the last step (u32), 9 words.
    DeviceBuf tlas;        // SceneBVH TLAS nodes (2 float4 each), as uploaded
    uint32_t tlasCount = 0;
    std::vector<float> hostTlas;
    DeviceBuf tests, post;
    bool testsOn = false;
    // Probabilistic policy (NOMAD_POLICY_PROBABILISTIC), host state of updateProbabilisticResidency
    bool probOn = false;
    std::vector<uint8_t> probDesired, probPending;
    std::vector<uint32_t> probPromoted, probDemoted, probDwell;
    std::vector<float> probEvidence;
    std::vector<uint32_t> probOrder;  // also the order of the environment policies
    // EnvironmentHit: render statistics at the previous step (segments, escapes)
    uint64_t prevSegments = 0, prevEscapes = 0;
    // EnergyImportance: last residency change per object (step number), smoothed importance,
    // static per-object importance and emitted power, the scene's total primitive importance
    std::vector<uint32_t> lastToggle;
    std::vector<float> energyHist, energyTotal, energyEmit;
    float energyPrimTotal = 0.0f;
    // DistanceLOD policy (NOMAD_POLICY_DISTANCE_LOD): object cooldowns and the last step's tests
    bool lodOn = false;
    std::vector<uint32_t> objCooldown;
    std::vector<float> lodDist;
    std::vector<uint8_t> lodFlags;
  } res;
  void *mlp = nullptr;  // MlpState (mlp.cu)
  // Geometry paging (paging.cu): the paged node layout's width (0 = off) and its state.
  uint32_t pagedWidth = 0;
  void *paging = nullptr;
  // Host mirror of the device residency flags after a device step: copied asynchronously into
  // pinned memory and applied to objResident / instances when a host call next needs them.
  bool resHostStale = false;
  uint8_t *resPinned = nullptr;
  size_t resPinnedBytes = 0;
  cudaEvent_t resEvent = nullptr;
  ~nomad_ctx() {
    if (resEvent) cudaEventDestroy(resEvent);
    if (resPinned) cudaFreeHost(resPinned);
  }
};

// Applies a pending device residency step to the host mirror (waits for its flag copy).
nomad_status nomad_residency_sync_host(nomad_ctx *ctx);
// Per-object "rays tested" of n closest-hit rays (2 float4 each) and their hits (5 words each;
// the count from lenDev when set), added to ctx->res.tests on the context's stream.
nomad_status nomad_build_shade_records(nomad_ctx *ctx, const float *materials, uint32_t primCount);
nomad_status nomad_count_object_tests(nomad_ctx *ctx, const float4 *rays, const int32_t *hits5, uint64_t n,
                                      const uint32_t *lenDev);
constexpr int kPostWords = 9;

void nomad_mlp_free(void *p);
void nomad_paging_free(nomad_ctx *ctx);
// Paging: the arena word of the triangle record at leaf position `pos` (-1 when its object is
// Cold), after updating the cold copy's activity word to `word`.
int64_t nomad_paging_record_word(nomad_ctx *ctx, uint32_t pos, int32_t word);
// Paging: the ref an object's TLAS link takes when it is resident (kEmptyRef until published).
int32_t nomad_paging_ref(const nomad_ctx *ctx, uint32_t obj);
// Paging: makes the context's stream wait for the copies queued so far.
nomad_status nomad_paging_order(nomad_ctx *ctx);
nomad_status nomad_mlp_infer_device(nomad_ctx *ctx, const float *X, uint64_t n, float *y);
namespace nomad_res {
struct FeatArgs;
}
// Learned policy: per-object features (as the feature kernel computes them) and MLP scores in one
// launch; keys[o] receives the score.
nomad_status nomad_mlp_score_objects(nomad_ctx *ctx, const nomad_res::FeatArgs *fa, float *keys);
// Whether the context holds a usable model (initialised, set, trained or loaded, not rejected).
bool nomad_mlp_ready(nomad_ctx *ctx);
// Residency device state: created at upload, mirrored after host-side flushes.
nomad_status nomad_residency_init(nomad_ctx *ctx);
nomad_status nomad_residency_mirror(nomad_ctx *ctx);
// Rebuilds the light CDF on the device if residency changed since the last build.
nomad_status nomad_lights_update(nomad_ctx *ctx);
// Rewrites every object's instance slot in the wide layouts from the device residency flags.
nomad_status nomad_patch_wide(nomad_ctx *ctx);
// Launches a closest- or any-hit trace of n device rays with traversal configuration `cfg`
// (queue length read from the device when lenDev is set).
nomad_status nomad_trace_variant(nomad_ctx *ctx, const nomad_traversal &cfg, bool any, const float4 *rays, uint64_t n,
                                 const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5,
                                 uint8_t *occ, uint32_t *counts, cudaStream_t st);
// The short-stack persistent kernels (trace_regroup.cu).
nomad_status nomad_trace_regroup(nomad_ctx *ctx, const nomad_traversal &cfg, bool any, const float4 *rays, uint64_t n,
                                 const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5, uint8_t *occ,
                                 uint32_t *counts, cudaStream_t s);
// Opts the short-stack kernels in to large dynamic shared memory (once per context creation).
cudaError_t nomad_regroup_init();
// Looks up (again) the device address of the allocation-free entry point's static scratch array
// on `device`, which must be current; called when a context is created on that device.
cudaError_t nomad_noalloc_lookup(int device);
// The hybrid packet kernels (trace_packet.cu).
nomad_status nomad_trace_packet(nomad_ctx *ctx, const nomad_traversal &cfg, bool any, const float4 *rays, uint64_t n,
                                const uint32_t *lenDev, unsigned long long *cursor, int32_t *hits5, uint8_t *occ,
                                uint32_t *counts, cudaStream_t s);
// NOMAD_KERNEL_* as a traversal configuration.
nomad_traversal nomad_kernel_config(uint32_t kernel);
// Whether `cfg` is valid and can run on the uploaded scene (stack depth, layout sizes).
bool nomad_traversal_ok(const nomad_ctx *ctx, const nomad_traversal &cfg, std::string *why);

inline nomad_status nomad_fail(nomad_ctx *c, nomad_status st, const std::string &msg) {
  if (c) c->err = msg;
  return st;
}

inline nomad_status nomad_cuda_fail(nomad_ctx *c, cudaError_t e, const char *what) {
  return nomad_fail(c, NOMAD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define NOMAD_CUDA(ctx, call)                                         \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) return nomad_cuda_fail(ctx, e_, #call);    \
  } while (0)

#define NOMAD_DEVICE_SCOPE(ctx)                                                  \
  NomadDeviceScope nomad_device_scope_((ctx)->device);                           \
  if (nomad_device_scope_.err != cudaSuccess)                                    \
  return nomad_cuda_fail(ctx, nomad_device_scope_.err, "cudaSetDevice")

