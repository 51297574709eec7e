// Builds the B200 traversal layout (pair nodes + leaf-ordered triangle records) from the
// SceneBVH arrays. See layout.h for the format.
#include "layout.h"

#include <algorithm>
#include <cstring>

#include "vec3.h"

namespace nomad {

namespace {
struct N2 {
  const float *p;
  float mn(int i) const { return p[i]; }
  float mx(int i) const { return p[4 + i]; }
  int32_t a() const { return float_bits_as_int(p[3]); }
  int32_t b() const { return float_bits_as_int(p[7]); }
};
}  // namespace

bool build_traversal_layout(const float *bvh, uint32_t bvhCount, const float *tlas,
                            uint32_t tlasCount, const float *prims, const int32_t *primIndices,
                            uint32_t primCount, const ObjectRange *objects, uint32_t objectCount,
                            TraversalLayout &out, std::vector<uint8_t> &resident,
                            std::string &err) {
  out = TraversalLayout();
  if (tlasCount == 0 || objectCount == 0 || primCount == 0) {
    err = "scene needs at least one TLAS node, object and primitive";
    return false;
  }
  auto bn = [&](uint32_t i) { return N2{bvh + 8ull * i}; };
  auto tn = [&](uint32_t i) { return N2{tlas + 8ull * i}; };

  // Objects and the primitive -> object map.
  out.primObject.assign(primCount, -1);
  for (uint32_t o = 0; o < objectCount; ++o) {
    uint64_t end = (uint64_t)objects[o].first + objects[o].count;
    if (end > primCount) {
      err = "instance record " + std::to_string(o) + " covers primitives past the end";
      return false;
    }
    for (uint64_t p = objects[o].first; p < end; ++p) {
      if (out.primObject[p] != -1) {
        err = "instance records overlap";
        return false;
      }
      out.primObject[p] = static_cast<int32_t>(o);
    }
  }

  // primIndices must be a permutation of [0, primCount).
  out.primPos.assign(primCount, -1);
  for (uint32_t k = 0; k < primCount; ++k) {
    int32_t p = primIndices[k];
    if (p < 0 || (uint32_t)p >= primCount || out.primPos[p] != -1) {
      err = "primitive index buffer is not a permutation";
      return false;
    }
    out.primPos[p] = static_cast<int32_t>(k);
  }

  // BLAS nodes: validate children and find roots (nodes nobody references). SceneBVH emits
  // children after their parent (pre-order); the compacted residency arrays emit them before
  // (post-order, Renderer.cpp:5513-5556). Either order is accepted, the same for every node,
  // which also rules out cycles.
  std::vector<uint8_t> isChild(bvhCount, 0);
  int childrenAfter = -1;  // 1 pre-order, 0 post-order, -1 not known yet
  for (uint32_t i = 0; i < bvhCount; ++i) {
    N2 n = bn(i);
    if (n.b() > 0) {
      int64_t first = n.a(), cnt = n.b();
      if (first < 0 || first + cnt > (int64_t)primCount) {
        err = "BLAS leaf " + std::to_string(i) + " range out of bounds";
        return false;
      }
    } else {
      int32_t l = n.a(), r = -n.b();
      if (childrenAfter < 0) childrenAfter = l > (int32_t)i ? 1 : 0;
      const bool ordered = childrenAfter ? (l > (int32_t)i && r > (int32_t)i) : (l >= 0 && r >= 0 && l < (int32_t)i && r < (int32_t)i);
      if (!ordered || (uint32_t)l >= bvhCount || (uint32_t)r >= bvhCount) {
        err = "BLAS node " + std::to_string(i) + " has an out-of-order or out-of-range child";
        return false;
      }
      if (isChild[l] || isChild[r]) {
        err = "BLAS node referenced twice";
        return false;
      }
      isChild[l] = isChild[r] = 1;
    }
  }
  out.blasPostOrder = childrenAfter == 0;
  std::vector<int32_t> roots;
  for (uint32_t i = 0; i < bvhCount; ++i)
    if (!isChild[i]) roots.push_back(static_cast<int32_t>(i));
  std::vector<int32_t> objRoot(objectCount, -1);
  size_t ri = 0;
  for (uint32_t o = 0; o < objectCount; ++o) {
    if (objects[o].count == 0) continue;
    if (ri >= roots.size()) {
      err = "fewer BLAS roots than non-empty objects";
      return false;
    }
    objRoot[o] = roots[ri++];
    if (objects[o].blasRoot >= 0 && objects[o].blasRoot != objRoot[o]) {
      err = "instance " + std::to_string(o) + " blas root does not match the node arrays";
      return false;
    }
  }
  if (ri != roots.size()) {
    err = "more BLAS roots than non-empty objects";
    return false;
  }

  // TLAS validation (pre-order, children after parent).
  for (uint32_t i = 0; i < tlasCount; ++i) {
    N2 n = tn(i);
    if (n.a() < 0) {
      int32_t o = -(n.a() + 1);
      // an empty object may stay in the TLAS when it is not resident (compacted arrays keep the
      // full scene's TLAS, Renderer.cpp:5756)
      if (o < 0 || (uint32_t)o >= objectCount || (objects[o].count == 0 && objects[o].blasRoot >= 0)) {
        err = "TLAS leaf " + std::to_string(i) + " names a bad object";
        return false;
      }
    } else if (n.a() <= (int32_t)i || n.b() <= (int32_t)i || (uint32_t)n.a() >= tlasCount ||
               (uint32_t)n.b() >= tlasCount) {
      err = "TLAS node " + std::to_string(i) + " has an out-of-order or out-of-range child";
      return false;
    }
  }

  // Pair-node numbering: TLAS internal nodes first, in breadth-first order from the root so the
  // top levels form a prefix that a kernel can stage in shared memory, then BLAS internal nodes.
  std::vector<int32_t> tPair(tlasCount, -1), bPair(bvhCount, -1);
  uint32_t np = 0;
  if (tn(0).a() >= 0) {
    std::vector<uint32_t> queue{0};
    std::vector<uint8_t> seen(tlasCount, 0);
    seen[0] = 1;
    for (size_t q = 0; q < queue.size(); ++q) {
      uint32_t i = queue[q];
      tPair[i] = static_cast<int32_t>(np++);
      N2 n = tn(i);
      for (int32_t c : {n.a(), n.b()}) {
        if (seen[c]) {
          err = "TLAS node " + std::to_string(c) + " referenced twice";
          return false;
        }
        seen[c] = 1;
        if (tn(c).a() >= 0) queue.push_back(static_cast<uint32_t>(c));
      }
    }
  }
  out.tlasPairCount = np;
  for (uint32_t i = 0; i < bvhCount; ++i)
    if (bn(i).b() <= 0) bPair[i] = static_cast<int32_t>(np++);
  if (np > 0x7ffffff0u) {
    err = "too many nodes";
    return false;
  }

  auto blasRef = [&](int32_t node) -> int32_t {
    N2 n = bn(node);
    return n.b() > 0 ? ~n.a() : bPair[node];
  };
  out.objBlasRef.assign(objectCount, kEmptyRef);
  out.objRootNode = objRoot;
  out.objSlot.assign(objectCount, -2);
  resident.assign(objectCount, 0);
  for (uint32_t o = 0; o < objectCount; ++o) {
    if (objRoot[o] >= 0) out.objBlasRef[o] = blasRef(objRoot[o]);
    resident[o] = (objects[o].blasRoot >= 0 && objects[o].count > 0) ? 1 : 0;
  }

  out.pnodes.assign(16ull * np, 0.0f);
  auto put_child = [&](uint32_t pair, int side, const N2 &box, int32_t ref) {
    float *p = out.pnodes.data() + 16ull * pair;
    float *mn = side == 0 ? p + 0 : p + 8;
    float *mx = side == 0 ? p + 4 : p + 12;
    for (int k = 0; k < 3; ++k) {
      mn[k] = box.mn(k);
      mx[k] = box.mx(k);
    }
    p[side == 0 ? 3 : 7] = int_bits_as_float(ref);
  };
  auto tlasChildRef = [&](uint32_t child, int64_t slot) -> int32_t {
    N2 c = tn(child);
    if (c.a() >= 0) return tPair[child];
    int32_t o = -(c.a() + 1);
    out.objSlot[o] = slot;
    return resident[o] ? out.objBlasRef[o] : kEmptyRef;
  };
  for (uint32_t i = 0; i < tlasCount; ++i) {
    N2 n = tn(i);
    if (n.a() < 0 || tPair[i] < 0) continue;  // leaf, or not reachable from the root
    uint32_t pr = static_cast<uint32_t>(tPair[i]);
    put_child(pr, 0, tn(n.a()), tlasChildRef(n.a(), 2ll * pr + 0));
    put_child(pr, 1, tn(n.b()), tlasChildRef(n.b(), 2ll * pr + 1));
  }
  for (uint32_t i = 0; i < bvhCount; ++i) {
    N2 n = bn(i);
    if (n.b() > 0) continue;
    uint32_t pr = static_cast<uint32_t>(bPair[i]);
    int32_t l = n.a(), r = -n.b();
    put_child(pr, 0, bn(l), blasRef(l));
    put_child(pr, 1, bn(r), blasRef(r));
  }
  N2 root = tn(0);
  for (int k = 0; k < 3; ++k) {
    out.rootMin[k] = root.mn(k);
    out.rootMax[k] = root.mx(k);
  }
  if (root.a() >= 0) {
    out.rootRef = 0;
  } else {
    int32_t o = -(root.a() + 1);
    out.objSlot[o] = -1;
    out.rootRef = resident[o] ? out.objBlasRef[o] : kEmptyRef;
  }
  for (uint32_t o = 0; o < objectCount; ++o) {
    if (objects[o].count > 0 && out.objSlot[o] == -2) {
      err = "object " + std::to_string(o) + " is missing from the TLAS";
      return false;
    }
  }

  // Leaf-ordered triangle records, with the leaf-closing flag.
  out.tris.assign(12ull * primCount, 0.0f);
  std::vector<uint8_t> closes(primCount, 0);
  for (uint32_t i = 0; i < bvhCount; ++i) {
    N2 n = bn(i);
    if (n.b() > 0) closes[n.a() + n.b() - 1] = 1;
  }
  for (uint32_t k = 0; k < primCount; ++k) {
    int32_t p = primIndices[k];
    const float *g = prims + 28ull * p;
    int type = static_cast<int>(g[3]);
    float *t = out.tris.data() + 12ull * k;
    V3 v0(g[0], g[1], g[2]), v1(g[4], g[5], g[6]), v2(g[8], g[9], g[10]);
    V3 a = v0, b, c;
    if (type == 1) {
      b = v1 - v0;  // edge1, as firstHitBVH computes it (Shaders/PathTracing.h:776-777)
      c = v2 - v0;
    } else {
      b = v1;  // rectangle u / sphere radius in .x
      c = v2;  // rectangle v
    }
    t[0] = a.x; t[1] = a.y; t[2] = a.z; t[3] = int_bits_as_float(p);
    t[4] = b.x; t[5] = b.y; t[6] = b.z; t[7] = int_bits_as_float(out.primObject[p]);
    t[8] = c.x; t[9] = c.y; t[10] = c.z;
    t[11] = int_bits_as_float(type | (closes[k] ? kLastInLeaf : 0));
  }
  // Leaves must tile [0, primCount) with no gaps so every chain of records ends at a flag.
  for (uint32_t o = 0; o < objectCount; ++o) {
    if (objects[o].count == 0) continue;
    uint32_t last = objects[o].first + objects[o].count - 1;
    if (!closes[last]) {
      err = "BLAS leaves do not tile object " + std::to_string(o);
      return false;
    }
  }

  // Depth of the combined tree (pair nodes on the longest path + 1 for the leaf).
  uint32_t depth = 0;
  if (out.rootRef != kEmptyRef || np > 0) {
    std::vector<std::pair<int32_t, uint32_t>> st;
    // Walk with all instances linked so the depth bound holds for any residency state.
    auto linked = [&](uint32_t pair, int side) -> int32_t {
      const float *p = out.pnodes.data() + 16ull * pair;
      int32_t ref = float_bits_as_int(p[side == 0 ? 3 : 7]);
      return ref;
    };
    std::vector<int32_t> slotObj(2ull * np, -1);
    for (uint32_t o = 0; o < objectCount; ++o)
      if (out.objSlot[o] >= 0) slotObj[out.objSlot[o]] = static_cast<int32_t>(o);
    int32_t r0 = root.a() >= 0 ? 0 : out.objBlasRef[-(root.a() + 1)];
    if (r0 != kEmptyRef) st.push_back({r0, 1});
    while (!st.empty()) {
      auto [ref, d] = st.back();
      st.pop_back();
      if (ref < 0) {
        depth = std::max(depth, d);
        continue;
      }
      depth = std::max(depth, d);
      for (int s = 0; s < 2; ++s) {
        int32_t c = linked(ref, s);
        int32_t so = slotObj[2ull * ref + s];
        if (so >= 0) c = out.objBlasRef[so];
        if (c != kEmptyRef) st.push_back({c, d + 1});
      }
    }
  }
  out.maxDepth = depth;
  return true;
}

}  // namespace nomad
