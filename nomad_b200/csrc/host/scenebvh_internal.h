// Internal: the SceneBVH data a handle owns, and the stages shared by the host builder
// (scenebvh.cpp) and the GPU BLAS builder (cuda/scenebvh_gpu.cu).
#pragma once
#include <cstdint>
#include <memory>
#include <utility>
#include <vector>

#include "../../../include/nomad_scene.h"
#include "vec3.h"

namespace nomad {

struct BNode {
  V3 mn, mx;
  int32_t leftFirst;
  int32_t count;  // > 0 leaf prim count; <= 0 -(right child)
};

// One object's BLAS in build (pre-) order; root = -1 for an empty object.
struct BlasResult {
  std::vector<BNode> nodes;
  int root = -1;
  uint32_t depth = 0;
};

// Allocator whose resize() leaves floats uninitialised, so that the threads that fill the
// packed primitive arrays also take their first-touch page faults in parallel.
template <typename T>
struct NoInitAlloc : std::allocator<T> {
  template <typename U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <typename U>
  NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
  template <typename U>
  void construct(U *p) noexcept {
    ::new (static_cast<void *>(p)) U;
  }
  template <typename U, typename... Args>
  void construct(U *p, Args &&...args) {
    ::new (static_cast<void *>(p)) U(std::forward<Args>(args)...);
  }
};

struct SceneBVHData {
  std::vector<float> bvh, tlas, objBounds;
  std::vector<float, NoInitAlloc<float>> prims, materials;  // every element written by pack_prims
  std::vector<int32_t> primIndices;
  std::vector<nomad_instance_record> instances;
  uint32_t primCount = 0, objectCount = 0, maxDepth = 0;
};

nomad_status scenebvh_validate(const nomad_scene_desc *d);
// Depths, concatenation with rebased children (SceneBVH.cpp:117-150), the TLAS and the packed
// arrays, from per-object BLAS results and the final primitive permutation.
nomad_status scenebvh_finish(const nomad_scene_desc *d, std::vector<BlasResult> &results,
                             const std::vector<int32_t> &indices, SceneBVHData &out,
                             uint32_t threads);
// createTransformsBuffer / createMaterialsBuffer packing on `threads` host threads (0 = all).
void pack_prims(const nomad_scene_desc &d, SceneBVHData &out, uint32_t threads);

}  // namespace nomad

struct nomad_scenebvh {
  nomad::SceneBVHData data;
};
