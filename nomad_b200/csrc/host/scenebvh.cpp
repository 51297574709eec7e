// SceneBVH-compatible host builder and GPU-buffer packer.
//
// Restates, in this project's own code, the algorithm of the reference's Scene::buildBVH
// (Nomad Path Tracer/Scene/SceneBVH.cpp:16-159):
//   * one binary BLAS per object, built by binned SAH (12 bins per axis, cost
//     0.125 + SA_L/SA_P*N_L + SA_R/SA_P*N_R, SceneBVH.cpp:704-815), leaf when the range
//     holds <= 8 primitives or the parent box has no area (:573-578), split position
//     taken from the winning bin's left count after a stable sort of the range on the
//     split axis centroid (:596-617);
//   * per-object node arrays concatenated in object order with child indices rebased
//     (:117-150);
//   * an object-level SAH TLAS (:625-702) whose leaves encode left = -(object+1),
//     right = object, with a median split when the parent box has no area or the SAH
//     finds no split.
// The layouts and the order of every floating-point operation follow the reference so the
// packed arrays match it bit for bit (checked against the reference's own SceneBVH.cpp in
// the test-suite).
#include "../../../include/nomad_scene.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <memory>
#include <new>
#include <numeric>
#include <thread>
#include <vector>

#include "scenebvh_internal.h"
#include "vec3.h"

namespace nomad {

namespace {

constexpr float kFrameEps = 1.0e-6f;  // Triangle.h:21 / Rectangle.h:20

V3 safe_normalize(V3 v) {
  float len = length(v);
  if (len > kFrameEps && finite3(v)) return v / len;
  return V3(0.0f, 0.0f, 0.0f);
}

// Per-primitive shading frame, restated from Triangle::computeFrame (Triangle.h:20-107).
void triangle_frame(V3 v0, V3 v1, V3 v2, float uv0x, float uv0y, float uv1x, float uv1y,
                    float uv2x, float uv2y, V3 &tangent, V3 &bitangent, V3 &normal) {
  V3 edge1 = v1 - v0;
  V3 edge2 = v2 - v0;
  V3 n = safe_normalize(cross(edge1, edge2));
  if (length(n) <= kFrameEps || !finite3(n)) n = V3(0.0f, 1.0f, 0.0f);

  float duv1x = uv1x - uv0x, duv1y = uv1y - uv0y;
  float duv2x = uv2x - uv0x, duv2y = uv2y - uv0y;
  float det = duv1x * duv2y - duv1y * duv2x;
  V3 t(0.0f, 0.0f, 0.0f), b(0.0f, 0.0f, 0.0f);
  if (std::fabs(det) > kFrameEps) {
    float invDet = 1.0f / det;
    t = safe_normalize((edge1 * duv2y - edge2 * duv1y) * invDet);
    b = safe_normalize((edge2 * duv1x - edge1 * duv2x) * invDet);
  }
  bool tValid = length(t) > kFrameEps && finite3(t);
  bool bValid = length(b) > kFrameEps && finite3(b);
  if (!tValid || !bValid) {
    t = safe_normalize(edge1);
    if (length(t) <= kFrameEps || !finite3(t)) t = safe_normalize(edge2);
    if (length(t) <= kFrameEps || !finite3(t)) {
      V3 up = std::fabs(n.y) < 0.999f ? V3(0.0f, 1.0f, 0.0f) : V3(1.0f, 0.0f, 0.0f);
      t = safe_normalize(cross(up, n));
    }
    if (length(t) <= kFrameEps || !finite3(t)) t = V3(1.0f, 0.0f, 0.0f);
    b = safe_normalize(cross(n, t));
    if (length(b) <= kFrameEps || !finite3(b)) b = safe_normalize(cross(t, n));
  } else {
    t = safe_normalize(t - n * dot(n, t));
    b = safe_normalize(b - n * dot(n, b));
  }
  if (length(b) <= kFrameEps || !finite3(b)) b = safe_normalize(cross(n, t));
  if (length(b) <= kFrameEps || !finite3(b)) b = V3(0.0f, 1.0f, 0.0f);
  tangent = t;
  bitangent = b;
  normal = safe_normalize(n);
  if (length(normal) <= kFrameEps || !finite3(normal)) normal = V3(0.0f, 0.0f, 1.0f);
}

// Restated from Rectangle::computeFrame (Rectangle.h:19-75). Returns supportsNormalMap.
bool rectangle_frame(V3 u, V3 v, V3 &tangent, V3 &bitangent, V3 &normal) {
  V3 t = safe_normalize(u);
  V3 b = safe_normalize(v);
  V3 n = safe_normalize(cross(t, b));
  if (length(t) <= kFrameEps || !finite3(t)) t = V3(1.0f, 0.0f, 0.0f);
  if (length(b) <= kFrameEps || !finite3(b)) {
    V3 ref = std::fabs(t.y) < 0.999f ? V3(0.0f, 1.0f, 0.0f) : V3(0.0f, 0.0f, 1.0f);
    b = safe_normalize(cross(ref, t));
  }
  if (length(n) <= kFrameEps || !finite3(n)) n = safe_normalize(cross(u, v));
  if (length(n) <= kFrameEps || !finite3(n)) n = V3(0.0f, 1.0f, 0.0f);
  t = safe_normalize(t - n * dot(n, t));
  b = safe_normalize(cross(n, t));
  bool tv = length(t) > kFrameEps && finite3(t);
  bool bv = length(b) > kFrameEps && finite3(b);
  bool nv = length(n) > kFrameEps && finite3(n);
  bool ok = tv && bv && nv;
  if (!ok) {
    t = V3(1.0f, 0.0f, 0.0f);
    b = V3(0.0f, 1.0f, 0.0f);
    n = V3(0.0f, 0.0f, 1.0f);
  }
  tangent = t;
  bitangent = b;
  normal = n;
  return ok;
}

struct Prim {
  int type;
  const float *g;  // NOMAD_PRIM_GEOM_FLOATS floats
  V3 a() const { return V3(g[0], g[1], g[2]); }
  V3 b() const { return V3(g[3], g[4], g[5]); }
  V3 c() const { return V3(g[6], g[7], g[8]); }
};

// primitiveBounds (SceneBVH.cpp:843-864).
void prim_bounds(const Prim &p, V3 &mn, V3 &mx) {
  if (p.type == NOMAD_PRIM_SPHERE) {
    float r = p.g[3];
    mn = p.a() - r;
    mx = p.a() + r;
  } else if (p.type == NOMAD_PRIM_RECTANGLE) {
    V3 c = p.a(), e1 = p.b(), e2 = p.c();
    V3 c1 = c - e1 - e2, c2 = c - e1 + e2, c3 = c + e1 - e2, c4 = c + e1 + e2;
    mn = vmin(vmin(c1, c2), vmin(c3, c4));
    mx = vmax(vmax(c1, c2), vmax(c3, c4));
  } else {
    mn = vmin(p.a(), vmin(p.b(), p.c()));
    mx = vmax(p.a(), vmax(p.b(), p.c()));
  }
}

// primitiveAxisValue (SceneBVH.cpp:822-830).
float prim_axis(const Prim &p, int axis) {
  if (p.type == NOMAD_PRIM_SPHERE) return p.g[axis];
  if (p.type == NOMAD_PRIM_RECTANGLE) return p.g[axis];
  return (p.g[axis] + p.g[3 + axis] + p.g[6 + axis]) / 3.0f;
}

float surface_area(V3 mn, V3 mx) {
  V3 d = mx - mn;
  return 2.0f * (d.x * d.y + d.y * d.z + d.z * d.x);
}

struct SahResult {
  int axis = -1;
  size_t leftCount = 0;
  float cost = std::numeric_limits<float>::max();
};

// Binned SAH over 12 bins per axis (SceneBVH.cpp:704-815).
SahResult sah_split(const V3 *mins, const V3 *maxs, const V3 *cents, size_t count,
                    float parentArea) {
  SahResult r;
  if (count <= 1 || parentArea <= 0.0f) return r;
  constexpr int kBins = 12;
  const float fmax = std::numeric_limits<float>::max();
  float cmin[3] = {fmax, fmax, fmax}, cmax[3] = {-fmax, -fmax, -fmax};
  for (size_t i = 0; i < count; ++i) {
    for (int a = 0; a < 3; ++a) {
      float c = cents[i][a];
      cmin[a] = std::min(cmin[a], c);
      cmax[a] = std::max(cmax[a], c);
    }
  }
  std::array<int, kBins> bc;
  std::array<V3, kBins> bmn, bmx, pmn, pmx, smn, smx;
  std::array<int, kBins> pc, sc;
  for (int axis = 0; axis < 3; ++axis) {
    float lo = cmin[axis], hi = cmax[axis];
    float range = hi - lo;
    if (range <= 1e-6f) continue;
    for (int i = 0; i < kBins; ++i) {
      bc[i] = 0;
      bmn[i] = V3(fmax);
      bmx[i] = V3(-fmax);
    }
    float inv = 1.0f / range;
    for (size_t i = 0; i < count; ++i) {
      float c = cents[i][axis];
      int bin = static_cast<int>((c - lo) * inv * kBins);
      bin = std::max(0, std::min(kBins - 1, bin));
      ++bc[bin];
      bmn[bin] = vmin(bmn[bin], mins[i]);
      bmx[bin] = vmax(bmx[bin], maxs[i]);
    }
    V3 rmn(fmax), rmx(-fmax);
    int rc = 0;
    for (int i = 0; i < kBins; ++i) {
      if (bc[i] > 0) {
        rmn = vmin(rmn, bmn[i]);
        rmx = vmax(rmx, bmx[i]);
      }
      rc += bc[i];
      pmn[i] = rmn;
      pmx[i] = rmx;
      pc[i] = rc;
    }
    rmn = V3(fmax);
    rmx = V3(-fmax);
    rc = 0;
    for (int i = kBins - 1; i >= 0; --i) {
      if (bc[i] > 0) {
        rmn = vmin(rmn, bmn[i]);
        rmx = vmax(rmx, bmx[i]);
      }
      rc += bc[i];
      smn[i] = rmn;
      smx[i] = rmx;
      sc[i] = rc;
    }
    for (int i = 0; i < kBins - 1; ++i) {
      int l = pc[i], rr = sc[i + 1];
      if (l == 0 || rr == 0) continue;
      float saL = surface_area(pmn[i], pmx[i]);
      float saR = surface_area(smn[i + 1], smx[i + 1]);
      float cost = 0.125f + (saL / parentArea) * l + (saR / parentArea) * rr;
      if (cost < r.cost) {
        r.cost = cost;
        r.axis = axis;
        r.leftCount = static_cast<size_t>(l);
      }
    }
  }
  return r;
}

struct BlasBuilder {
  const std::vector<Prim> &prims;
  std::vector<int64_t> &indices;  // global primitive permutation (primitiveIndices)
  std::vector<BNode> nodes;       // local node array of one object
  std::vector<V3> mins, maxs, cents;

  BlasBuilder(const std::vector<Prim> &p, std::vector<int64_t> &idx) : prims(p), indices(idx) {}

  // buildBVHRecursive (SceneBVH.cpp:549-623)
  int build(size_t start, size_t end) {
    const float fmax = std::numeric_limits<float>::max();
    V3 bMin(fmax), bMax(-fmax);
    for (size_t i = start; i < end; ++i) {
      V3 mn, mx;
      prim_bounds(prims[indices[i]], mn, mx);
      bMin = vmin(bMin, mn);
      bMax = vmax(bMax, mx);
    }
    BNode node;
    node.mn = bMin;
    node.mx = bMax;
    node.leftFirst = static_cast<int32_t>(start);
    size_t range = end - start;
    node.count = static_cast<int32_t>(range);
    int idx = static_cast<int>(nodes.size());
    nodes.push_back(node);
    if (node.count <= 8) return idx;
    float parentArea = surface_area(bMin, bMax);
    if (parentArea <= 0.0f) return idx;
    mins.resize(range);
    maxs.resize(range);
    cents.resize(range);
    for (size_t i = start; i < end; ++i) {
      const Prim &p = prims[indices[i]];
      V3 mn, mx;
      prim_bounds(p, mn, mx);
      mins[i - start] = mn;
      maxs[i - start] = mx;
      cents[i - start] = V3(prim_axis(p, 0), prim_axis(p, 1), prim_axis(p, 2));
    }
    SahResult s = sah_split(mins.data(), maxs.data(), cents.data(), range, parentArea);
    int axis = s.axis;
    size_t leftCount = axis == -1 ? range / 2 : std::min(s.leftCount, range - 1);
    if (axis == -1 || leftCount == 0 || leftCount >= range) return idx;
    std::stable_sort(indices.begin() + start, indices.begin() + end,
                     [&](int64_t a, int64_t b) {
                       return prim_axis(prims[a], axis) < prim_axis(prims[b], axis);
                     });
    size_t split = start + leftCount;
    int l = build(start, split);
    int r = build(split, end);
    nodes[idx].leftFirst = l;
    nodes[idx].count = -r;
    return idx;
  }
};

struct TNode {
  V3 mn, mx;
  int32_t left = -1, right = -1;
};

struct TlasBuilder {
  const std::vector<V3> &objMin, &objMax;
  std::vector<int64_t> &objIdx;
  std::vector<TNode> nodes;

  float axis_value(int64_t o, int axis) const {
    return 0.5f * (objMin[o][axis] + objMax[o][axis]);
  }

  // buildTLASRecursive (SceneBVH.cpp:625-702)
  int build(size_t start, size_t end) {
    const float fmax = std::numeric_limits<float>::max();
    V3 bMin(fmax), bMax(-fmax);
    for (size_t i = start; i < end; ++i) {
      bMin = vmin(bMin, objMin[objIdx[i]]);
      bMax = vmax(bMax, objMax[objIdx[i]]);
    }
    TNode n;
    n.mn = bMin;
    n.mx = bMax;
    int idx = static_cast<int>(nodes.size());
    nodes.push_back(n);
    size_t range = end - start;
    if (range == 1) {
      int64_t o = objIdx[start];
      nodes[idx].left = -static_cast<int32_t>(o) - 1;
      nodes[idx].right = static_cast<int32_t>(o);
      return idx;
    }
    float parentArea = surface_area(bMin, bMax);
    auto median = [&]() {
      size_t mid = start + range / 2;
      int l = build(start, mid);
      int r = build(mid, end);
      nodes[idx].left = l;
      nodes[idx].right = r;
      return idx;
    };
    if (parentArea <= 0.0f) return median();
    std::vector<V3> mins(range), maxs(range), cents(range);
    for (size_t i = 0; i < range; ++i) {
      int64_t o = objIdx[start + i];
      mins[i] = objMin[o];
      maxs[i] = objMax[o];
      cents[i] = 0.5f * (objMin[o] + objMax[o]);
    }
    SahResult s = sah_split(mins.data(), maxs.data(), cents.data(), range, parentArea);
    int axis = s.axis;
    size_t leftCount = axis == -1 ? range / 2 : std::min(s.leftCount, range - 1);
    if (axis == -1 || leftCount == 0 || leftCount >= range) return median();
    size_t split = start + leftCount;
    std::sort(objIdx.begin() + start, objIdx.begin() + end,
              [&](int64_t a, int64_t b) { return axis_value(a, axis) < axis_value(b, axis); });
    int l = build(start, split);
    int r = build(split, end);
    nodes[idx].left = l;
    nodes[idx].right = r;
    return idx;
  }
};

}  // namespace

namespace {

void pack_range(const nomad_scene_desc &d, SceneBVHData &out, size_t lo, size_t hi) {
  for (size_t i = lo; i < hi; ++i) {
    const float *g = d.prim_geom + i * NOMAD_PRIM_GEOM_FLOATS;
    float *o = out.prims.data() + i * 28;
    for (int k = 0; k < 28; ++k) o[k] = 0.0f;
    int type = d.prim_type[i];
    auto put = [&](int slot, V3 v, float w) {
      o[slot * 4 + 0] = v.x;
      o[slot * 4 + 1] = v.y;
      o[slot * 4 + 2] = v.z;
      o[slot * 4 + 3] = w;
    };
    if (type == NOMAD_PRIM_SPHERE) {
      put(0, V3(g[0], g[1], g[2]), 0.0f);
      put(1, V3(g[3], 0, 0), 0.0f);
      put(6, V3(0.0f, 0.0f, 1.0f), 0.0f);
    } else if (type == NOMAD_PRIM_RECTANGLE) {
      V3 t, b, nn;
      bool ok = rectangle_frame(V3(g[3], g[4], g[5]), V3(g[6], g[7], g[8]), t, b, nn);
      put(0, V3(g[0], g[1], g[2]), 2.0f);
      put(1, V3(g[3], g[4], g[5]), 0.0f);
      put(2, V3(g[6], g[7], g[8]), 0.0f);
      put(4, t, 0.0f);
      put(5, b, 0.0f);
      put(6, nn, ok ? 1.0f : 0.0f);
    } else {
      V3 v0(g[0], g[1], g[2]), v1(g[3], g[4], g[5]), v2(g[6], g[7], g[8]);
      V3 t, b, nn;
      triangle_frame(v0, v1, v2, g[9], g[10], g[11], g[12], g[13], g[14], t, b, nn);
      put(0, v0, 1.0f);
      put(1, v1, g[9]);
      put(2, v2, g[10]);
      o[12] = g[11];
      o[13] = g[12];
      o[14] = g[13];
      o[15] = g[14];
      put(4, t, 0.0f);
      put(5, b, 0.0f);
      put(6, nn, 1.0f);
    }
    // createMaterialsBuffer / encodeMaterial (Material.h:32-44). Texture indices are
    // carried as floats already; they round-trip through int like the reference.
    const float *m = d.prim_material + i * NOMAD_MATERIAL_FLOATS;
    float *om = out.materials.data() + i * 20;
    for (int k = 0; k < 16; ++k) om[k] = m[k];
    om[16] = static_cast<float>(static_cast<int>(m[16]));
    om[17] = static_cast<float>(static_cast<int>(m[17]));
    om[18] = static_cast<float>(static_cast<int>(m[18]));
    om[19] = m[19];
  }
}

}  // namespace

void pack_prims(const nomad_scene_desc &d, SceneBVHData &out, uint32_t threads) {
  // createTransformsBuffer (SceneBVH.cpp:165-209) after the per-primitive frame set-up
  // done by Scene::addObjectInternal (Scene.cpp:137-146). Every primitive is packed on its
  // own, so the range is split over host threads.
  const size_t n = d.prim_count;
  out.prims.resize(n * 28);
  out.materials.resize(n * 20);
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t chunk = 65536;
  const size_t nt = std::min<size_t>(threads ? threads : hw, (n + chunk - 1) / chunk);
  if (nt <= 1) {
    pack_range(d, out, 0, n);
    return;
  }
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (;;) {
      const size_t lo = next.fetch_add(chunk);
      if (lo >= n) break;
      pack_range(d, out, lo, std::min(n, lo + chunk));
    }
  };
  std::vector<std::thread> pool;
  for (size_t t = 0; t < nt; ++t) pool.emplace_back(worker);
  for (auto &t : pool) t.join();
}

// Runs fn(lo, hi) over [0, n) in chunks on up to `threads` host threads (0 = all); each index is
// visited by exactly one call, so work that writes only its own indices gives the same result
// for any thread count.
template <class F>
static void parallel_chunks(size_t n, size_t chunk, uint32_t threads, F &&fn) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t nt = std::min<size_t>(threads ? threads : hw, (n + chunk - 1) / chunk);
  if (nt <= 1) {
    if (n) fn(size_t(0), n);
    return;
  }
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (;;) {
      const size_t lo = next.fetch_add(chunk);
      if (lo >= n) break;
      fn(lo, std::min(n, lo + chunk));
    }
  };
  std::vector<std::thread> pool;
  for (size_t t = 1; t < nt; ++t) pool.emplace_back(worker);
  worker();
  for (auto &t : pool) t.join();
}

nomad_status scenebvh_validate(const nomad_scene_desc *d) {
  if (!d || d->prim_count == 0 || d->object_count == 0) return NOMAD_ERR_INVALID_ARGUMENT;
  if (!d->prim_type || !d->prim_geom || !d->prim_material || !d->object_first ||
      !d->object_prims)
    return NOMAD_ERR_INVALID_ARGUMENT;
  if (d->prim_count > 0x7fffffffu / 8u) return NOMAD_ERR_LIMIT;
  uint64_t expect = 0;
  for (uint32_t o = 0; o < d->object_count; ++o) {
    if (d->object_first[o] != expect) return NOMAD_ERR_SCENE_INVALID;
    expect += d->object_prims[o];
  }
  if (expect != d->prim_count) return NOMAD_ERR_SCENE_INVALID;
  std::atomic<bool> bad{false};
  parallel_chunks(d->prim_count, 1 << 16, 0, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi && !bad.load(std::memory_order_relaxed); ++i) {
      int t = d->prim_type[i];
      bool ok = t == NOMAD_PRIM_SPHERE || t == NOMAD_PRIM_TRIANGLE || t == NOMAD_PRIM_RECTANGLE;
      const float *g = d->prim_geom + i * NOMAD_PRIM_GEOM_FLOATS;
      for (int k = 0; k < 9 && ok; ++k) ok = std::isfinite(g[k]);
      if (!ok) bad.store(true, std::memory_order_relaxed);
    }
  });
  return bad.load() ? NOMAD_ERR_SCENE_INVALID : NOMAD_OK;
}

static nomad_status build_impl(const nomad_scene_desc *d, uint32_t threads, SceneBVHData &out) {
  nomad_status st = scenebvh_validate(d);
  if (st != NOMAD_OK) return st;
  const size_t n = d->prim_count;
  const size_t nobj = d->object_count;
  std::vector<Prim> prims(n);
  for (size_t i = 0; i < n; ++i) prims[i] = Prim{d->prim_type[i], d->prim_geom + i * NOMAD_PRIM_GEOM_FLOATS};
  std::vector<int64_t> indices(n);
  std::iota(indices.begin(), indices.end(), 0);

  std::vector<BlasResult> results(nobj);
  std::atomic<size_t> next{0};
  auto worker = [&]() {
    for (;;) {
      size_t o = next.fetch_add(1);
      if (o >= nobj) break;
      if (d->object_prims[o] == 0) continue;
      BlasBuilder b(prims, indices);
      b.nodes.reserve(d->object_prims[o] * 2);
      size_t first = d->object_first[o];
      results[o].root = b.build(first, first + d->object_prims[o]);
      results[o].nodes = std::move(b.nodes);
    }
  };
  unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  unsigned nt = threads ? threads : hw;
  nt = std::max(1u, std::min<unsigned>(nt, static_cast<unsigned>(nobj)));
  if (nt == 1) {
    worker();
  } else {
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; ++t) pool.emplace_back(worker);
    for (auto &t : pool) t.join();
  }
  std::vector<int32_t> idx32(n);
  for (size_t i = 0; i < n; ++i) idx32[i] = static_cast<int32_t>(indices[i]);
  return scenebvh_finish(d, results, idx32, out, threads);
}

// Everything after the per-object BLAS builds: BLAS depths, concatenation with rebased
// children, the TLAS, and the packed arrays.
nomad_status scenebvh_finish(const nomad_scene_desc *d, std::vector<BlasResult> &results,
                             const std::vector<int32_t> &indices, SceneBVHData &out,
                             uint32_t threads) {
  const size_t n = d->prim_count;
  const size_t nobj = d->object_count;
  // depth of every BLAS (iterative, nodes only), one object per task
  parallel_chunks(nobj, 16, threads, [&](size_t lo, size_t hi) {
    std::vector<std::pair<int, uint32_t>> st;
    for (size_t o = lo; o < hi; ++o) {
      BlasResult &r = results[o];
      if (r.root < 0) continue;
      st.assign(1, {r.root, 1u});
      uint32_t depth = 0;
      while (!st.empty()) {
        auto [ni, dd] = st.back();
        st.pop_back();
        depth = std::max(depth, dd);
        const BNode &nd = r.nodes[ni];
        if (nd.count <= 0) {
          st.push_back({nd.leftFirst, dd + 1});
          st.push_back({-nd.count, dd + 1});
        }
      }
      r.depth = depth;
    }
  });

  // Concatenation with rebased children (SceneBVH.cpp:117-150): each object's nodes go to
  // [base, base + size) of the packed array, base the node count of the objects before it.
  std::vector<size_t> base(nobj, 0);
  size_t total = 0;
  for (size_t o = 0; o < nobj; ++o) {
    base[o] = total;
    if (results[o].root >= 0) total += results[o].nodes.size();
  }
  if (total > 0x7fffffffu) return NOMAD_ERR_LIMIT;
  std::vector<int32_t> blasRoot(nobj, -1);
  std::vector<V3> objMin(nobj, V3(0.0f)), objMax(nobj, V3(0.0f));
  std::vector<int64_t> objIdx;
  for (size_t o = 0; o < nobj; ++o) {
    const BlasResult &r = results[o];
    if (r.root < 0) continue;
    blasRoot[o] = static_cast<int32_t>(base[o]) + r.root;
    objMin[o] = r.nodes[r.root].mn;
    objMax[o] = r.nodes[r.root].mx;
    objIdx.push_back(static_cast<int64_t>(o));
  }
  out.bvh.resize(total * 8);
  parallel_chunks(nobj, 4, threads, [&](size_t lo, size_t hi) {
    for (size_t o = lo; o < hi; ++o) {
      const BlasResult &r = results[o];
      if (r.root < 0) continue;
      const int32_t b = static_cast<int32_t>(base[o]);
      float *p = out.bvh.data() + base[o] * 8;
      for (const BNode &nd : r.nodes) {
        int32_t lf = nd.leftFirst, cnt = nd.count;
        if (cnt < 0) {
          lf += b;
          cnt = -(-cnt + b);
        }
        p[0] = nd.mn.x; p[1] = nd.mn.y; p[2] = nd.mn.z;
        p[3] = int_bits_as_float(lf);
        p[4] = nd.mx.x; p[5] = nd.mx.y; p[6] = nd.mx.z;
        p[7] = int_bits_as_float(cnt);
        p += 8;
      }
    }
  });

  TlasBuilder tb{objMin, objMax, objIdx, {}};
  if (!objIdx.empty()) tb.build(0, objIdx.size());

  // Depth: TLAS depth of each leaf + that object's BLAS depth.
  uint32_t maxDepth = 0;
  if (!tb.nodes.empty()) {
    std::vector<std::pair<int, uint32_t>> st{{0, 1u}};
    while (!st.empty()) {
      auto [ni, dd] = st.back();
      st.pop_back();
      const TNode &nd = tb.nodes[ni];
      if (nd.left < 0) {
        maxDepth = std::max(maxDepth, dd + results[nd.right].depth);
      } else {
        st.push_back({nd.left, dd + 1});
        st.push_back({nd.right, dd + 1});
      }
    }
  }

  out.primCount = static_cast<uint32_t>(n);
  out.objectCount = static_cast<uint32_t>(nobj);
  out.maxDepth = maxDepth;
  out.tlas.resize(tb.nodes.size() * 8);
  for (size_t i = 0; i < tb.nodes.size(); ++i) {
    float *p = out.tlas.data() + i * 8;
    const TNode &t = tb.nodes[i];
    p[0] = t.mn.x; p[1] = t.mn.y; p[2] = t.mn.z; p[3] = int_bits_as_float(t.left);
    p[4] = t.mx.x; p[5] = t.mx.y; p[6] = t.mx.z; p[7] = int_bits_as_float(t.right);
  }
  out.primIndices.assign(indices.begin(), indices.begin() + static_cast<std::ptrdiff_t>(n));
  out.instances.resize(nobj);
  out.objBounds.resize(nobj * 6);
  for (size_t o = 0; o < nobj; ++o) {
    nomad_instance_record r;
    r.blas_root_index = blasRoot[o];
    r.primitive_base = d->object_first[o];
    r.primitive_count = d->object_prims[o];
    r.primitive_index_base = d->object_first[o];
    out.instances[o] = r;
    float *b = out.objBounds.data() + o * 6;
    b[0] = objMin[o].x; b[1] = objMin[o].y; b[2] = objMin[o].z;
    b[3] = objMax[o].x; b[4] = objMax[o].y; b[5] = objMax[o].z;
  }
  pack_prims(*d, out, threads);
  return NOMAD_OK;
}

}  // namespace nomad

extern "C" nomad_status nomad_scenebvh_build(const nomad_scene_desc *desc, uint32_t threads,
                                             nomad_scenebvh **out) {
  if (!out) return NOMAD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  try {
    std::unique_ptr<nomad_scenebvh> h(new nomad_scenebvh());
    nomad_status st = nomad::build_impl(desc, threads, h->data);
    if (st != NOMAD_OK) return st;
    *out = h.release();
    return NOMAD_OK;
  } catch (const std::bad_alloc &) {
    return NOMAD_ERR_OUT_OF_MEMORY;
  } catch (...) {
    return NOMAD_ERR_INVALID_ARGUMENT;
  }
}

extern "C" nomad_status nomad_scenebvh_view_get(const nomad_scenebvh *h, nomad_scenebvh_view *v) {
  if (!h || !v) return NOMAD_ERR_INVALID_ARGUMENT;
  const auto &d = h->data;
  v->prim_count = d.primCount;
  v->object_count = d.objectCount;
  v->bvh_node_count = static_cast<uint32_t>(d.bvh.size() / 8);
  v->tlas_node_count = static_cast<uint32_t>(d.tlas.size() / 8);
  v->bvh_nodes = d.bvh.data();
  v->tlas_nodes = d.tlas.data();
  v->prims = d.prims.data();
  v->materials = d.materials.data();
  v->prim_indices = d.primIndices.data();
  v->instances = d.instances.data();
  v->object_bounds = d.objBounds.data();
  v->max_depth = d.maxDepth;
  return NOMAD_OK;
}

extern "C" void nomad_scenebvh_free(nomad_scenebvh *h) { delete h; }
