// Internal: the libnomad_rt context shared by the traversal (rt_core.cu) and the path tracer
// (pathtrace.cu) translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../../include/nomad_rt.h"
#include "../host/layout.h"
#include "rt_device.cuh"

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
};

// Light-sampling tables over the active emissive primitives, restated from the light CDF build
// of Renderer::rebuildResidentResources (Renderer.cpp:5161-5211).
struct LightTables {
  std::vector<uint32_t> indices;  // primitive index of each light
  std::vector<float> cdf;         // running sum of area * emission strength
  std::vector<float> pdfLookup;   // per primitive: weight / total (0 for non-lights)
  float total = 0.0f;
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
  DeviceBuf lightIdx, lightCdf, lightPdf;
  uint32_t lightCount = 0;
  float lightTotal = 0.0f;
  bool lightsDirty = true;
  // ReSTIR DI reservoirs (current and previous frame) and surface records
  DeviceBuf resv[2], surf[2];
  uint64_t restirPixels = 0;
  int restirCur = 0;
  bool restirValid = false;
};

struct nomad_ctx {
  int device = 0;
  int smCount = 0;
  cudaStream_t stream = nullptr;     // stream used by calls (own or caller's)
  cudaStream_t ownStream = nullptr;
  cudaStream_t copyStreams[2] = {nullptr, nullptr};
  std::string err;
  uint32_t kernel = NOMAD_KERNEL_BVH2;
  bool sceneReady = false;
  // scene sizes
  uint32_t primCount = 0, objectCount = 0;
  // device memory
  DeviceBuf arena;      // pair nodes then triangle records
  DeviceBuf prims, materials;
  DeviceBuf objHits, status, cursor;
  DeviceBuf stageIn, stageOut, stageAux;  // host-pointer staging
  DeviceBuf patchOffs, patchVals;
  size_t pnodeWords = 0;  // int32 words of the pair-node part of the arena
  nomad_dev::DevScene scene{};
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
};

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

// Rebuilds the light tables from the host copies of the scene and the active set.
void nomad_build_lights(const nomad_ctx *ctx, LightTables &out);
