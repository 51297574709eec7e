// ORACLE — test infrastructure only (the checker, never the product).
//
// Scalar restatement of the reference's compacted resident-geometry rebuild, the branch of
// Renderer::rebuildResidentResources taken when residency compaction is on
// (Nomad Path Tracer/Renderer/Renderer.cpp:5359-5560, the cached-BLAS path). For every object,
// in object order:
//   * its primitives are visited in the BLAS leaf order of the object's cached BLAS
//     (cachedPrimitiveIndices, filled by Scene::buildBVH, SceneBVH.cpp:78-97); each active one
//     gets the next compact index, its packed primitive and material are appended, the remap
//     entry (compact -> global) is pushed, and the compact primitive index is its own compact
//     index (:5411-5497);
//   * an object with no active primitive gets primitiveCount 0 and blasRootIndex -1 (:5500-5508);
//   * otherwise its cached BLAS is rewritten bottom-up (rebuildNode, :5513-5556): a leaf keeps
//     its bounds, starts at the compact index of its first active primitive and counts its
//     active primitives, or disappears when none is active; an inner node disappears when both
//     children did and is replaced by its surviving child when one did; surviving nodes are
//     appended after their children (post-order) and rebased to the object's first compact node
//     (:5558-5577); the instance's root is the rebuilt root (:5560-5562).
// The TLAS is reused unchanged (:5756). primitive_to_resident maps a global primitive to its
// compact index, -1 when inactive (reset at :4967, set at :5425).
//
// Works directly on the concatenated SceneBVH arrays: a cached BLAS is the object's node range
// with object-local indices, which is the same tree read with global indices.
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

struct Node {
  float mn[3];
  int32_t leftFirst;
  float mx[3];
  int32_t count;
};

Node load_node(const float *bvh, int32_t i) {
  Node n;
  const float *p = bvh + (size_t)i * 8;
  n.mn[0] = p[0]; n.mn[1] = p[1]; n.mn[2] = p[2];
  std::memcpy(&n.leftFirst, p + 3, 4);
  n.mx[0] = p[4]; n.mx[1] = p[5]; n.mx[2] = p[6];
  std::memcpy(&n.count, p + 7, 4);
  return n;
}

struct Ctx {
  const float *bvh;
  uint32_t nodeCount;
  const std::vector<int32_t> *remap;  // leaf position -> object-local compact index or -1
  uint32_t first;                     // the object's first leaf position
  uint32_t indexBase;                 // record.primitiveIndexBase
  std::vector<Node> rebuilt;
};

// rebuildNode (Renderer.cpp:5513-5556), indices global.
int32_t rebuild(Ctx &c, int32_t idx) {
  if (idx < 0 || (uint32_t)idx >= c.nodeCount) return -1;
  Node a = load_node(c.bvh, idx);
  if (a.count > 0) {
    int32_t newFirst = -1, newCount = 0;
    for (int32_t i = 0; i < a.count; ++i) {
      const int64_t local = (int64_t)a.leftFirst + i - (int64_t)c.first;
      if (local < 0 || (size_t)local >= c.remap->size()) continue;
      const int32_t r = (*c.remap)[(size_t)local];
      if (r < 0) continue;
      if (newFirst < 0) newFirst = (int32_t)(c.indexBase + (uint32_t)r);
      ++newCount;
    }
    if (newCount == 0) return -1;
    a.leftFirst = newFirst;
    a.count = newCount;
  } else {
    const int32_t l = rebuild(c, a.leftFirst);
    const int32_t r = rebuild(c, -a.count);
    if (l < 0 && r < 0) return -1;
    if (l < 0) return r;
    if (r < 0) return l;
    a.leftFirst = l;
    a.count = -r;
  }
  c.rebuilt.push_back(a);
  return (int32_t)c.rebuilt.size() - 1;
}

}  // namespace

extern "C" int oracle_compact(const float *bvh, uint32_t nodeCount, const float *prims, const float *mats,
                              const int32_t *primIdx, uint32_t primCount, const int32_t *inst /* 4 per object */,
                              uint32_t objectCount, const uint8_t *active, float *oBvh, float *oPrims, float *oMats,
                              int32_t *oIdx, uint32_t *oRemap, int32_t *oPrimToRes, int32_t *oInst,
                              uint32_t *oCounts /* [0] primitives, [1] nodes */) {
  for (uint32_t g = 0; g < primCount; ++g) oPrimToRes[g] = -1;
  uint32_t nPrim = 0, nNode = 0;
  std::vector<int32_t> remap;
  for (uint32_t o = 0; o < objectCount; ++o) {
    const int32_t root = inst[o * 4 + 0];
    const uint32_t first = (uint32_t)inst[o * 4 + 1], count = (uint32_t)inst[o * 4 + 2];
    int32_t *rec = oInst + o * 4;
    rec[0] = -1;
    rec[1] = (int32_t)nPrim;  // primitiveBase = remapUpload.size()
    rec[3] = (int32_t)nPrim;  // primitiveIndexBase = compactPrimitiveIndices.size()
    rec[2] = 0;
    if (root < 0 || count == 0) continue;  // no cached BLAS and no primitive
    const uint32_t indexBase = nPrim;
    remap.assign(count, -1);
    uint32_t activeCount = 0;
    for (uint32_t local = 0; local < count; ++local) {
      const int32_t g = primIdx[first + local];
      if (g < 0 || (uint32_t)g >= primCount || !active[g]) continue;
      remap[local] = (int32_t)activeCount;
      const uint32_t k = nPrim + activeCount;
      oRemap[k] = (uint32_t)g;
      oPrimToRes[g] = (int32_t)k;
      std::memcpy(oPrims + (size_t)k * 28, prims + (size_t)g * 28, 28 * 4);
      std::memcpy(oMats + (size_t)k * 20, mats + (size_t)g * 20, 20 * 4);
      oIdx[k] = (int32_t)k;
      ++activeCount;
    }
    rec[2] = (int32_t)activeCount;
    if (activeCount == 0) continue;
    Ctx c{bvh, nodeCount, &remap, first, indexBase, {}};
    const int32_t rootNew = rebuild(c, root);
    nPrim += activeCount;
    if (rootNew < 0) continue;  // cannot happen with activeCount > 0
    const uint32_t nodeBase = nNode;
    rec[0] = (int32_t)(nodeBase + (uint32_t)rootNew);
    for (Node a : c.rebuilt) {
      if (a.count <= 0) {
        const int32_t l = a.leftFirst + (int32_t)nodeBase;
        const int32_t r = -a.count + (int32_t)nodeBase;
        a.leftFirst = l;
        a.count = -r;
      }
      float *p = oBvh + (size_t)nNode * 8;
      p[0] = a.mn[0]; p[1] = a.mn[1]; p[2] = a.mn[2];
      std::memcpy(p + 3, &a.leftFirst, 4);
      p[4] = a.mx[0]; p[5] = a.mx[1]; p[6] = a.mx[2];
      std::memcpy(p + 7, &a.count, 4);
      ++nNode;
    }
  }
  oCounts[0] = nPrim;
  oCounts[1] = nNode;
  return 0;
}
