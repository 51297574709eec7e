// ORACLE — test infrastructure only. Internals of the scalar contract traversal shared by
// contract.cpp (ray queries) and pathtrace.cpp (the scalar path tracer). See contract.cpp for
// the reference file:line map and the contract.
#pragma once
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace oracle_core {
namespace {

const float RAY_EPS = 1e-4f;
const float PRUNE = 1.0009765625f;

struct F3 {
  float x, y, z;
};
inline F3 mk(float x, float y, float z) { return F3{x, y, z}; }
inline F3 sub(F3 a, F3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float dot(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross(F3 a, F3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline bool finite(F3 v) { return std::isfinite(v.x) && std::isfinite(v.y) && std::isfinite(v.z); }
inline F3 normalize(F3 v) {
  float l = std::sqrt(dot(v, v));
  return mk(v.x / l, v.y / l, v.z / l);
}
inline int32_t fbits(float f) {
  int32_t i;
  std::memcpy(&i, &f, 4);
  return i;
}
inline float comp(F3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }

struct Ray {
  F3 o, d;
  float tmax;
};

struct Scene {
  const float *bvh;
  const float *tlas;
  uint32_t tlasCount;
  const float *prims;
  const int32_t *primIndices;
  const uint8_t *active;
  const int32_t *blasRoot;  // per object, < 0 = not resident
  const int32_t *primObject;
};

// intersectAABB: slab over [tMin, tMax]; |d| < RAY_EPS axes test the origin only.
bool aabb(const Ray &r, const float *mn, const float *mx, float tMin, float tMax, float *tEntry) {
  for (int i = 0; i < 3; ++i) {
    float dir = comp(r.d, i), o = comp(r.o, i);
    if (std::fabs(dir) < RAY_EPS) {
      if (o < mn[i] || o > mx[i]) return false;
      continue;
    }
    float invD = 1.0f / dir;
    float t0 = (mn[i] - o) * invD;
    float t1 = (mx[i] - o) * invD;
    if (invD < 0.0f) std::swap(t0, t1);
    tMin = std::max(tMin, t0);
    tMax = std::min(tMax, t1);
    if (tMax < tMin) return false;
  }
  if (tEntry) *tEntry = tMin;
  return true;
}

struct Hit {
  float t, u, v;
  int32_t prim, inst;
};

// One primitive test; accepts when RAY_EPS < t and (t, prim) beats (best.t, best.prim).
bool test_prim(const Scene &s, const Ray &r, int32_t p, Hit &best) {
  const float *g = s.prims + 28ll * p;
  int type = static_cast<int>(g[3]);
  float tt, bu = 0.0f, bv = 0.0f;
  if (type == 1) {
    F3 v0 = mk(g[0], g[1], g[2]), v1 = mk(g[4], g[5], g[6]), v2 = mk(g[8], g[9], g[10]);
    F3 e1 = sub(v1, v0), e2 = sub(v2, v0);
    F3 h = cross(r.d, e2);
    float a = dot(e1, h);
    if (!(std::fabs(a) > 1e-5f)) return false;
    float f = 1.0f / a;
    F3 sv = sub(r.o, v0);
    float u = f * dot(sv, h);
    if (!(u >= 0.0f && u <= 1.0f)) return false;
    F3 q = cross(sv, e1);
    float v = f * dot(r.d, q);
    if (!(v >= 0.0f && u + v <= 1.0f)) return false;
    tt = f * dot(e2, q);
    bu = u;
    bv = v;
  } else if (type == 2) {
    F3 c = mk(g[0], g[1], g[2]), e1 = mk(g[4], g[5], g[6]), e2 = mk(g[8], g[9], g[10]);
    F3 fb = cross(e1, e2);
    float fl = dot(fb, fb);
    F3 n = (fl > RAY_EPS && finite(fb)) ? normalize(fb) : mk(0.0f, 1.0f, 0.0f);
    F3 sn = mk(g[24], g[25], g[26]);
    if (dot(sn, sn) > RAY_EPS && finite(sn)) n = normalize(sn);
    float denom = dot(n, r.d);
    if (!(std::fabs(denom) > 1e-5f)) return false;
    tt = dot(sub(c, r.o), n) / denom;
    if (!(tt > RAY_EPS)) return false;
    F3 hp = mk(r.o.x + tt * r.d.x, r.o.y + tt * r.d.y, r.o.z + tt * r.d.z);
    F3 rel = sub(hp, c);
    float u = dot(rel, e1) / dot(e1, e1);
    float v = dot(rel, e2) / dot(e2, e2);
    if (!(std::fabs(u) <= 1.0f && std::fabs(v) <= 1.0f)) return false;
  } else if (type == 0) {
    F3 c = mk(g[0], g[1], g[2]);
    float radius = g[4];
    F3 oc = sub(r.o, c);
    float a = dot(r.d, r.d);
    float b = dot(oc, r.d);
    float cc = dot(oc, oc) - radius * radius;
    float disc = b * b - a * cc;
    if (!(disc > 0.0f)) return false;
    tt = (-b - std::sqrt(disc)) / a;
  } else {
    return false;
  }
  if (!(tt > RAY_EPS)) return false;
  if (!(tt < best.t || (tt == best.t && best.prim >= 0 && p < best.prim))) return false;
  best.t = tt;
  best.u = bu;
  best.v = bv;
  best.prim = p;
  best.inst = s.primObject[p];
  return true;
}

struct Counters {
  uint32_t nodes = 0, tests = 0, insts = 0;
};

// Leaf of a BLAS: primitives primitiveIndices[first .. first+count).
// Returns true when ANY-mode found a hit.
template <bool ANY>
bool leaf(const Scene &s, const Ray &r, int32_t first, int32_t count, Hit &best, Counters *c) {
  for (int32_t i = 0; i < count; ++i) {
    int32_t p = s.primIndices[first + i];
    if (c) c->tests++;
    if (!s.active[p]) continue;
    if (test_prim(s, r, p, best) && ANY) return true;
  }
  return false;
}

inline float bound_of(const Hit &best, bool any, float tmax) {
  return any ? tmax : best.t * PRUNE;
}

// Reference order: TLAS children near-first by dot(centre - o, d) (PathTracing.h:1025-1062),
// BLAS fixed order (left pushed first, right popped first, :938-941); box tested at pop.
template <bool ANY>
void trace_reference_order(const Scene &s, const Ray &r, Hit &best) {
  struct E {
    int tl;  // 1 TLAS, 0 BLAS
    int32_t node;
  };
  std::vector<E> st;
  st.push_back({1, 0});
  float tmax = r.tmax;
  while (!st.empty()) {
    E e = st.back();
    st.pop_back();
    float bound = bound_of(best, ANY, tmax);
    if (e.tl) {
      const float *n = s.tlas + 8ll * e.node;
      if (!aabb(r, n, n + 4, RAY_EPS, bound, nullptr)) continue;
      int32_t l = fbits(n[3]), rr = fbits(n[7]);
      if (l < 0) {
        int32_t obj = -(l + 1);
        if (s.blasRoot[obj] >= 0) st.push_back({0, s.blasRoot[obj]});
        continue;
      }
      const float *ln = s.tlas + 8ll * l, *rn = s.tlas + 8ll * rr;
      F3 lc = mk((ln[0] + ln[4]) * 0.5f, (ln[1] + ln[5]) * 0.5f, (ln[2] + ln[6]) * 0.5f);
      F3 rc = mk((rn[0] + rn[4]) * 0.5f, (rn[1] + rn[5]) * 0.5f, (rn[2] + rn[6]) * 0.5f);
      float lk = dot(sub(lc, r.o), r.d), rk = dot(sub(rc, r.o), r.d);
      if (lk < rk) {
        st.push_back({1, rr});
        st.push_back({1, l});
      } else {
        st.push_back({1, l});
        st.push_back({1, rr});
      }
      continue;
    }
    const float *n = s.bvh + 8ll * e.node;
    if (!aabb(r, n, n + 4, RAY_EPS, bound, nullptr)) continue;
    int32_t lf = fbits(n[3]), second = fbits(n[7]);
    if (second > 0) {
      if (leaf<ANY>(s, r, lf, second, best, nullptr) && ANY) return;
    } else {
      st.push_back({0, lf});
      st.push_back({0, -second});
    }
  }
}

// Near-first order over the same binary arrays, mirroring a pair-node walk: an internal node
// tests both child boxes, descends into the nearer and defers the farther. A TLAS leaf reads the
// instance record and continues at that object's BLAS root without re-testing its box (the
// root box equals the TLAS leaf box). Counts box tests, primitive tests and instance reads.
template <bool ANY>
void trace_near_first(const Scene &s, const Ray &r, Hit &best, Counters *c) {
  // ref: kind 0 = TLAS node, 1 = BLAS node
  struct R {
    int kind;
    int32_t node;
  };
  float tmax = r.tmax;
  if (c) c->nodes++;
  if (!aabb(r, s.tlas, s.tlas + 4, RAY_EPS, bound_of(best, ANY, tmax), nullptr)) return;
  std::vector<R> st;
  auto resolve = [&](int kind, int32_t node, R &out) -> bool {
    // Follow TLAS leaves into their BLAS roots; false when the instance is not resident.
    if (kind == 0) {
      const float *n = s.tlas + 8ll * node;
      int32_t l = fbits(n[3]);
      if (l < 0) {
        if (c) c->insts++;
        int32_t obj = -(l + 1);
        if (s.blasRoot[obj] < 0) return false;
        out = R{1, s.blasRoot[obj]};
        return true;
      }
    }
    out = R{kind, node};
    return true;
  };
  R cur;
  if (!resolve(0, 0, cur)) return;
  for (;;) {
    const float *n = (cur.kind == 0 ? s.tlas : s.bvh) + 8ll * cur.node;
    bool isLeaf = cur.kind == 1 && fbits(n[7]) > 0;
    if (!isLeaf) {
      int32_t l = fbits(n[3]);
      int32_t rr = cur.kind == 0 ? fbits(n[7]) : -fbits(n[7]);
      const float *base = cur.kind == 0 ? s.tlas : s.bvh;
      const float *ln = base + 8ll * l, *rn = base + 8ll * rr;
      float bound = bound_of(best, ANY, tmax);
      float tl = 0, tr = 0;
      bool hl = aabb(r, ln, ln + 4, RAY_EPS, bound, &tl);
      bool hr = aabb(r, rn, rn + 4, RAY_EPS, bound, &tr);
      if (c) c->nodes += 2;
      R lref{}, rref{};
      if (hl) hl = resolve(cur.kind, l, lref);
      if (hr) hr = resolve(cur.kind, rr, rref);
      if (hl && hr) {
        bool lf = !(tr < tl);
        st.push_back(lf ? rref : lref);
        cur = lf ? lref : rref;
        continue;
      } else if (hl) {
        cur = lref;
        continue;
      } else if (hr) {
        cur = rref;
        continue;
      }
    } else {
      if (leaf<ANY>(s, r, fbits(n[3]), fbits(n[7]), best, c) && ANY) return;
    }
    if (st.empty()) return;
    cur = st.back();
    st.pop_back();
  }
}

// Brute force: every BLAS leaf whose box (and therefore every ancestor box) the ray enters
// within [RAY_EPS, tmax]; no pruning, so the result cannot depend on order.
template <bool ANY>
void trace_brute(const Scene &s, const Ray &r, Hit &best, uint32_t objectCount) {
  for (uint32_t o = 0; o < objectCount; ++o) {
    if (s.blasRoot[o] < 0) continue;
    std::vector<int32_t> st{s.blasRoot[o]};
    while (!st.empty()) {
      int32_t ni = st.back();
      st.pop_back();
      const float *n = s.bvh + 8ll * ni;
      if (!aabb(r, n, n + 4, RAY_EPS, r.tmax, nullptr)) continue;
      int32_t lf = fbits(n[3]), second = fbits(n[7]);
      if (second > 0) {
        if (leaf<ANY>(s, r, lf, second, best, nullptr) && ANY) return;
      } else {
        st.push_back(lf);
        st.push_back(-second);
      }
    }
  }
}

struct Job {
  Scene s;
  const float *rays;
  uint64_t n;
  int mode;
  bool any;
  uint32_t objectCount;
  float *hitsOut;     // closest: 5 words per ray (inst, prim as int bits; t, u, v)
  uint8_t *anyOut;
  uint32_t *work;     // 4 per ray
};

void run_range(const Job &j, uint64_t b, uint64_t e) {
  for (uint64_t i = b; i < e; ++i) {
    const float *q = j.rays + 8 * i;
    Ray r{mk(q[0], q[1], q[2]), mk(q[4], q[5], q[6]), q[7]};
    Hit h{r.tmax, 0.0f, 0.0f, -1, -1};
    Counters c;
    if (r.tmax > RAY_EPS) {
      if (j.any) {
        if (j.mode == 0) trace_reference_order<true>(j.s, r, h);
        else if (j.mode == 1) trace_near_first<true>(j.s, r, h, nullptr);
        else trace_brute<true>(j.s, r, h, j.objectCount);
      } else {
        if (j.mode == 0) trace_reference_order<false>(j.s, r, h);
        else if (j.mode == 1) trace_near_first<false>(j.s, r, h, j.work ? &c : nullptr);
        else trace_brute<false>(j.s, r, h, j.objectCount);
      }
    } else if (j.work) {
      c.nodes = 0;
    }
    if (j.any) {
      j.anyOut[i] = h.prim >= 0 ? 1 : 0;
    } else if (j.hitsOut) {
      int32_t *o = reinterpret_cast<int32_t *>(j.hitsOut + 5 * i);
      bool hit = h.prim >= 0;
      o[0] = hit ? h.inst : -1;
      o[1] = hit ? h.prim : -1;
      float t = hit ? h.t : INFINITY;
      std::memcpy(o + 2, &t, 4);
      float u = hit ? h.u : 0.0f, v = hit ? h.v : 0.0f;
      std::memcpy(o + 3, &u, 4);
      std::memcpy(o + 4, &v, 4);
    }
    if (j.work) {
      // A ray whose tmax excludes everything still tests the root box in the product.
      if (!(r.tmax > RAY_EPS)) c.nodes = 0;
      j.work[4 * i + 0] = c.nodes;
      j.work[4 * i + 1] = c.tests;
      j.work[4 * i + 2] = c.insts;
      j.work[4 * i + 3] = h.prim >= 0 ? 1u : 0u;
    }
  }
}

[[maybe_unused]] void run(const Job &j, uint32_t threads) {
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  if (threads == 1 || j.n < 1024) {
    run_range(j, 0, j.n);
    return;
  }
  std::atomic<uint64_t> next{0};
  const uint64_t chunk = 256;
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        uint64_t b = next.fetch_add(chunk);
        if (b >= j.n) break;
        run_range(j, b, std::min(j.n, b + chunk));
      }
    });
  for (auto &t : pool) t.join();
}

}  // namespace
}  // namespace oracle_core
