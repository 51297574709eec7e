// Collapses the binary pair-node layout into a 4- or 8-wide layout for the wide traversal
// kernels.
//
// A wide node holds up to W child boxes (structure-of-arrays: min x[W], min y[W], min z[W],
// max x[W], max y[W], max z[W]) and W child refs, padded to a multiple of 64 bytes (W = 4:
// 128 B, W = 8: 256 B). Children are gathered greedily: starting from a binary node's two
// children, the internal child with the largest surface area is replaced by its own two children
// until W children are reached. Every child box is a box of the binary tree, unchanged, so the
// set of primitives a ray can reach is the binary tree's (a box test of a child implies its
// ancestors' tests pass). The collapse never crosses an instance link (a TLAS leaf pointing to
// a BLAS root), so each object keeps exactly one slot to patch when its residency changes.
#include <algorithm>
#include <cmath>
#include <limits>

#include "layout.h"
#include "vec3.h"

namespace nomad {

namespace {

struct Child {
  float mn[3], mx[3];
  int32_t ref;      // pair-layout ref (internal pair index, leaf, or empty)
  int32_t object;   // >= 0 when this child is an instance link of that object
};

float area(const Child &c) {
  float dx = c.mx[0] - c.mn[0], dy = c.mx[1] - c.mn[1], dz = c.mx[2] - c.mn[2];
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

struct Builder {
  const TraversalLayout &L;
  WideLayout &W;
  int width;
  std::vector<int32_t> slotObj;  // pair slot -> object (instance links)

  Child child(uint32_t pair, int side) const {
    const float *p = L.pnodes.data() + 16ull * pair;
    Child c;
    const float *mn = side == 0 ? p + 0 : p + 8;
    const float *mx = side == 0 ? p + 4 : p + 12;
    for (int k = 0; k < 3; ++k) {
      c.mn[k] = mn[k];
      c.mx[k] = mx[k];
    }
    c.ref = float_bits_as_int(p[side == 0 ? 3 : 7]);
    c.object = slotObj[2ull * pair + side];
    return c;
  }

  // Builds the wide node rooted at pair node `pair`; returns its wide index.
  int32_t build(uint32_t pair) {
    std::vector<Child> kids = {child(pair, 0), child(pair, 1)};
    while ((int)kids.size() < width) {
      int best = -1;
      float bestA = -1.0f;
      for (int i = 0; i < (int)kids.size(); ++i) {
        const Child &c = kids[i];
        if (c.object >= 0 || c.ref < 0) continue;  // links, leaves and empty slots stay
        float a = area(c);
        if (a > bestA) {
          bestA = a;
          best = i;
        }
      }
      if (best < 0) break;
      uint32_t pr = static_cast<uint32_t>(kids[best].ref);
      Child a = child(pr, 0), b = child(pr, 1);
      kids[best] = a;
      kids.push_back(b);
    }
    int32_t idx = static_cast<int32_t>(W.nodes.size() / W.floatsPerNode);
    W.nodes.resize(W.nodes.size() + W.floatsPerNode, 0.0f);
    std::vector<int32_t> refs(width, kEmptyRef);
    for (int i = 0; i < (int)kids.size(); ++i) {
      const Child &c = kids[i];
      if (c.object >= 0) {
        W.objSlot[c.object] = (int64_t)idx * width + i;
        refs[i] = c.ref == kEmptyRef ? kEmptyRef : W.objBlasRef[c.object];
      } else if (c.ref >= 0) {
        refs[i] = build(static_cast<uint32_t>(c.ref));
      } else {
        refs[i] = c.ref;  // leaf (~first) or empty
      }
    }
    float *n = W.nodes.data() + (size_t)idx * W.floatsPerNode;
    const float inf = std::numeric_limits<float>::infinity();
    for (int i = 0; i < width; ++i) {
      bool used = i < (int)kids.size();
      for (int k = 0; k < 3; ++k) {
        n[k * width + i] = used ? kids[i].mn[k] : inf;
        n[(3 + k) * width + i] = used ? kids[i].mx[k] : -inf;
      }
      n[6 * width + i] = int_bits_as_float(refs[i]);
    }
    return idx;
  }
};

uint32_t wide_depth(const WideLayout &W, int32_t ref) {
  if (ref < 0) return ref == kEmptyRef ? 0 : 1;
  const float *n = W.nodes.data() + (size_t)ref * W.floatsPerNode;
  uint32_t d = 0;
  for (uint32_t i = 0; i < W.width; ++i) d = std::max(d, wide_depth(W, float_bits_as_int(n[6 * W.width + i])));
  return d + 1;
}

// Renumbers the nodes so the TLAS part (nodes reachable from the root without crossing an
// instance link) comes first in breadth-first order, followed by the BLAS nodes in build order.
// The top levels then form a prefix [0, tlasNodes) that a kernel can stage in shared memory.
void reorder_tlas_first(WideLayout &W) {
  const size_t fpn = W.floatsPerNode, nn = W.nodes.size() / fpn;
  if (W.rootRef < 0 || nn == 0) return;
  std::vector<uint8_t> isLink(nn * W.width, 0);
  for (int64_t s : W.objSlot)
    if (s >= 0) isLink[s] = 1;
  std::vector<int32_t> perm(nn, -1), order;
  order.reserve(nn);
  order.push_back(W.rootRef);
  perm[W.rootRef] = 0;
  for (size_t q = 0; q < order.size(); ++q) {
    const float *n = W.nodes.data() + (size_t)order[q] * fpn;
    for (uint32_t i = 0; i < W.width; ++i) {
      int32_t c = float_bits_as_int(n[6 * W.width + i]);
      if (c < 0 || isLink[(size_t)order[q] * W.width + i] || perm[c] >= 0) continue;
      perm[c] = static_cast<int32_t>(order.size());
      order.push_back(c);
    }
  }
  W.tlasNodes = static_cast<uint32_t>(order.size());
  for (size_t i = 0; i < nn; ++i)
    if (perm[i] < 0) {
      perm[i] = static_cast<int32_t>(order.size());
      order.push_back(static_cast<int32_t>(i));
    }
  std::vector<float> nodes(W.nodes.size());
  for (size_t k = 0; k < nn; ++k) {
    const float *src = W.nodes.data() + (size_t)order[k] * fpn;
    float *dst = nodes.data() + k * fpn;
    std::copy(src, src + fpn, dst);
    for (uint32_t i = 0; i < W.width; ++i) {
      int32_t c = float_bits_as_int(dst[6 * W.width + i]);
      if (c >= 0) dst[6 * W.width + i] = int_bits_as_float(perm[c]);
    }
  }
  W.nodes.swap(nodes);
  W.rootRef = perm[W.rootRef];
  for (int32_t &r : W.objBlasRef)
    if (r >= 0) r = perm[r];
  for (int64_t &s : W.objSlot)
    if (s >= 0) s = (int64_t)perm[s / W.width] * W.width + s % W.width;
}

}  // namespace

void build_wide_layout(const TraversalLayout &L, int width, const std::vector<uint8_t> &resident, WideLayout &W) {
  W = WideLayout();
  W.width = static_cast<uint32_t>(width);
  W.floatsPerNode = width == 4 ? 32 : 64;
  const size_t nobj = L.objBlasRef.size();
  W.objBlasRef.assign(nobj, kEmptyRef);
  W.objSlot.assign(nobj, -2);
  Builder b{L, W, width, {}};
  b.slotObj.assign(L.pnodes.size() / 16 * 2, -1);
  for (size_t o = 0; o < nobj; ++o)
    if (L.objSlot[o] >= 0) b.slotObj[L.objSlot[o]] = static_cast<int32_t>(o);
  // BLAS wide roots first (every object, resident or not, so it can come back later)
  for (size_t o = 0; o < nobj; ++o) {
    int32_t r = L.objBlasRef[o];
    W.objBlasRef[o] = r >= 0 ? b.build(static_cast<uint32_t>(r)) : r;
  }
  if (L.tlasPairCount > 0) {
    W.rootRef = b.build(0);
  } else {
    for (size_t o = 0; o < nobj; ++o)
      if (L.objSlot[o] == -1) {
        W.objSlot[o] = -1;
        W.rootRef = resident[o] ? W.objBlasRef[o] : kEmptyRef;
      }
  }
  reorder_tlas_first(W);
  // depth with every instance linked (bounds the stack for any residency state)
  uint32_t d = 0;
  if (L.tlasPairCount > 0) {
    // TLAS part plus the deepest BLAS below it
    uint32_t blas = 0;
    for (size_t o = 0; o < nobj; ++o) blas = std::max(blas, wide_depth(W, W.objBlasRef[o]));
    WideLayout tmp;  // depth of the TLAS part alone
    (void)tmp;
    uint32_t tl = 0;
    std::vector<std::pair<int32_t, uint32_t>> st{{W.rootRef, 1}};
    std::vector<uint8_t> isLink(W.nodes.size() / W.floatsPerNode * W.width, 0);
    for (size_t o = 0; o < nobj; ++o)
      if (W.objSlot[o] >= 0) isLink[W.objSlot[o]] = 1;
    while (!st.empty()) {
      auto [ref, dd] = st.back();
      st.pop_back();
      tl = std::max(tl, dd);
      if (ref < 0) continue;
      const float *n = W.nodes.data() + (size_t)ref * W.floatsPerNode;
      for (uint32_t i = 0; i < W.width; ++i) {
        if (isLink[(size_t)ref * W.width + i]) continue;
        int32_t c = float_bits_as_int(n[6 * W.width + i]);
        if (c >= 0) st.push_back({c, dd + 1});
      }
    }
    d = tl + blas;
  } else {
    d = wide_depth(W, W.rootRef);
  }
  W.maxDepth = d;
}

}  // namespace nomad
