// Traversal layout derived from the SceneBVH arrays.
//
// SceneBVH (Nomad Path Tracer/Scene/SceneBVH.cpp:420-488) stores one box per node, so a
// traversal must fetch both children to order them. The B200 layout stores, for every internal
// node of the TLAS and of every BLAS, the boxes of its two children in one 64-byte "pair node"
// (four float4, one aligned 64 B line), and the triangles in leaf order as 48-byte records
// holding v0 and the two edges (three float4). Because instances carry no transform
// (Renderer/Shaders/Structs.h:31-37), a TLAS leaf links straight to its object's BLAS root and
// the two levels form one tree walked by one loop.
//
// Pair node, four float4:
//   [0] left.min.xyz,  bits(left ref)      [1] left.max.xyz,  bits(right ref)
//   [2] right.min.xyz, 0                    [3] right.max.xyz, 0
// Child ref: >= 0 internal pair node index; kEmptyRef a non-resident instance (skipped);
// otherwise a leaf whose first triangle record is ~ref.
// Triangle record, three float4:
//   [0] v0.xyz, bits(prim)   prim < 0 (stored as ~prim) when the primitive is inactive
//   [1] e1.xyz, bits(instance)
//   [2] e2.xyz, bits(type | kLastInLeaf when it closes its leaf)
// For rectangles [0..2] hold center, u, v; for spheres center and radius (in [1].x); the
// kernel reads their stored normal from the packed primitive array when needed.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace nomad {

constexpr int32_t kEmptyRef = INT32_MIN;
constexpr int32_t kLastInLeaf = 1 << 8;

struct TraversalLayout {
  std::vector<float> pnodes;   // 16 floats per pair node
  std::vector<float> tris;     // 12 floats per triangle record
  float rootMin[3], rootMax[3];
  int32_t rootRef = kEmptyRef;
  uint32_t tlasPairCount = 0;  // pair nodes [0, tlasPairCount) belong to the TLAS
  uint32_t maxDepth = 0;       // longest root-to-leaf chain of pair nodes plus the leaf
  bool blasPostOrder = false;  // BLAS children stored before their parent (compacted arrays)
  // Per object: BLAS ref used when resident, and where the TLAS stores it:
  // slot = pairIndex * 2 + side (side 0 left, 1 right); -1 when the object is the TLAS root.
  std::vector<int32_t> objBlasRef;
  std::vector<int32_t> objRootNode;  // SceneBVH node index of each object's BLAS root, or -1
  std::vector<int64_t> objSlot;
  std::vector<int32_t> primObject;  // object of every primitive
  std::vector<int32_t> primPos;     // position of every primitive in leaf order
};

// 4- or 8-wide layout collapsed from the pair nodes (see wide.cpp). Leaves use the same
// triangle records; refs are encoded as in the pair layout.
struct WideLayout {
  uint32_t width = 0;
  uint32_t floatsPerNode = 0;        // 32 (W = 4) or 64 (W = 8)
  std::vector<float> nodes;
  int32_t rootRef = kEmptyRef;
  std::vector<int32_t> objBlasRef;   // wide ref of each object's BLAS root
  std::vector<int64_t> objSlot;      // node * W + k of each instance link, -1 root, -2 none
  uint32_t maxDepth = 0;             // wide nodes on the longest path (+1 for the leaf)
  uint32_t tlasNodes = 0;            // nodes [0, tlasNodes) are the TLAS part, breadth-first
};

void build_wide_layout(const TraversalLayout &L, int width, const std::vector<uint8_t> &resident, WideLayout &W);

struct ObjectRange {
  int32_t blasRoot;  // SceneObject::blasRootIndex, or -1 when the caller marks it non-resident
  uint32_t first, count;
};

// Builds the layout; returns false and sets `err` when the SceneBVH arrays are inconsistent
// (out-of-range children, cycles, bad leaf ranges, a primitive index repeated or missing).
// The BLAS root of every object is recovered from the node arrays (per-object node blocks are
// concatenated in object order, SceneBVH.cpp:122-150), so objects uploaded with
// blasRoot = -1 can become resident later. `resident[o]` receives the initial state.
bool build_traversal_layout(const float *bvh, uint32_t bvhCount, const float *tlas,
                            uint32_t tlasCount, const float *prims, const int32_t *primIndices,
                            uint32_t primCount, const ObjectRange *objects, uint32_t objectCount,
                            TraversalLayout &out, std::vector<uint8_t> &resident,
                            std::string &err);

}  // namespace nomad
