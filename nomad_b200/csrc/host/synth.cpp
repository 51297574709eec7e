// Seeded synthetic scenes: icosphere instances and a procedural city.
//
// They stand in for the reference's XML/OBJ scenes (Nomad Path Tracer/Scene/SceneLoader.cpp),
// keeping its convention that every instance is baked into world space at load time
// (SceneLoader.cpp:742-787) so each object owns its own world-space BLAS and the TLAS
// instance record carries no transform (Renderer/Shaders/Structs.h:31-37).
//
// Determinism: a splitmix64 stream drives every choice; geometry is computed in double and
// rounded to float once, so the same seed gives the same arrays on every x86-64 host with
// this toolchain.
#include "../../../include/nomad_scene.h"

#include <algorithm>
#include <cmath>
#include <map>
#include <memory>
#include <new>
#include <vector>

namespace nomad {
namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed ^ 0x9E3779B97F4A7C15ull) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  double normal() {
    double u1 = std::max(uniform(), 1e-300), u2 = uniform();
    return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
  }
};

struct D3 {
  double x, y, z;
};
inline D3 operator+(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 operator-(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 operator*(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 dnorm(D3 a) {
  double l = std::sqrt(ddot(a, a));
  return l > 0 ? a * (1.0 / l) : a;
}
inline D3 dcross(D3 a, D3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

struct Builder {
  std::vector<int32_t> type;
  std::vector<float> geom, mat;
  std::vector<uint32_t> objFirst, objPrims;
  uint32_t curFirst = 0;

  void begin_object() { curFirst = static_cast<uint32_t>(type.size()); }
  void end_object() {
    uint32_t cnt = static_cast<uint32_t>(type.size()) - curFirst;
    if (cnt == 0) return;
    objFirst.push_back(curFirst);
    objPrims.push_back(cnt);
  }
  void push_material(const float m[20]) { mat.insert(mat.end(), m, m + 20); }
  void tri(D3 a, D3 b, D3 c, const float m[20]) {
    type.push_back(NOMAD_PRIM_TRIANGLE);
    float g[15] = {(float)a.x, (float)a.y, (float)a.z, (float)b.x, (float)b.y, (float)b.z,
                   (float)c.x, (float)c.y, (float)c.z, 0, 0, 0, 0, 0, 0};
    geom.insert(geom.end(), g, g + 15);
    push_material(m);
  }
  void rect(D3 c, D3 u, D3 v, const float m[20]) {
    type.push_back(NOMAD_PRIM_RECTANGLE);
    float g[15] = {(float)c.x, (float)c.y, (float)c.z, (float)u.x, (float)u.y, (float)u.z,
                   (float)v.x, (float)v.y, (float)v.z, 0, 0, 0, 0, 0, 0};
    geom.insert(geom.end(), g, g + 15);
    push_material(m);
  }
};

// A material in the reference encoding (Material.h:32-44), untextured.
void make_material(float out[20], D3 diffuse, D3 specular, float shininess, D3 emission,
                   float power, float roughness) {
  float m[20] = {(float)diffuse.x, (float)diffuse.y, (float)diffuse.z, 1.0f,
                 (float)specular.x, (float)specular.y, (float)specular.z, shininess,
                 (float)emission.x, (float)emission.y, (float)emission.z, power,
                 0.0f, 0.0f, 0.0f, 1.0f,
                 -1.0f, -1.0f, -1.0f, roughness};
  std::copy(m, m + 20, out);
}

// Icosahedron subdivided `levels` times, projected to the unit sphere.
void icosphere(int levels, std::vector<D3> &verts, std::vector<int> &tris) {
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  verts = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
           {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
  for (auto &v : verts) v = dnorm(v);
  tris = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4,
          11, 10, 2, 10, 7, 6, 7, 1, 8, 3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8,
          3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
  for (int l = 0; l < levels; ++l) {
    std::map<std::pair<int, int>, int> mid;
    auto midpoint = [&](int a, int b) {
      auto key = std::make_pair(std::min(a, b), std::max(a, b));
      auto it = mid.find(key);
      if (it != mid.end()) return it->second;
      D3 m = dnorm((verts[a] + verts[b]) * 0.5);
      verts.push_back(m);
      int idx = static_cast<int>(verts.size()) - 1;
      mid[key] = idx;
      return idx;
    };
    std::vector<int> nt;
    for (size_t i = 0; i < tris.size(); i += 3) {
      int a = tris[i], b = tris[i + 1], c = tris[i + 2];
      int ab = midpoint(a, b), bc = midpoint(b, c), ca = midpoint(c, a);
      int add[12] = {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca};
      nt.insert(nt.end(), add, add + 12);
    }
    tris.swap(nt);
  }
}

// Uniform random rotation from a unit quaternion (Shoemake's method).
void random_rotation(Rng &r, double m[9]) {
  double u1 = r.uniform(), u2 = r.uniform(), u3 = r.uniform();
  double a = std::sqrt(1 - u1), b = std::sqrt(u1);
  double qx = a * std::sin(6.283185307179586 * u2), qy = a * std::cos(6.283185307179586 * u2);
  double qz = b * std::sin(6.283185307179586 * u3), qw = b * std::cos(6.283185307179586 * u3);
  m[0] = 1 - 2 * (qy * qy + qz * qz); m[1] = 2 * (qx * qy - qz * qw); m[2] = 2 * (qx * qz + qy * qw);
  m[3] = 2 * (qx * qy + qz * qw); m[4] = 1 - 2 * (qx * qx + qz * qz); m[5] = 2 * (qy * qz - qx * qw);
  m[6] = 2 * (qx * qz - qy * qw); m[7] = 2 * (qy * qz + qx * qw); m[8] = 1 - 2 * (qx * qx + qy * qy);
}

// Hash-based 3-D value noise in [-1, 1] with smoothstep interpolation.
double hash3(int64_t x, int64_t y, int64_t z, uint64_t seed) {
  uint64_t h = seed ^ (uint64_t)x * 0x8DA6B343ull ^ (uint64_t)y * 0xD8163841ull ^
               (uint64_t)z * 0xCB1AB31Full;
  h ^= h >> 33;
  h *= 0xFF51AFD7ED558CCDull;
  h ^= h >> 33;
  h *= 0xC4CEB9FE1A85EC53ull;
  h ^= h >> 33;
  return (h >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}
double value_noise(D3 p, uint64_t seed) {
  double fx = std::floor(p.x), fy = std::floor(p.y), fz = std::floor(p.z);
  int64_t ix = (int64_t)fx, iy = (int64_t)fy, iz = (int64_t)fz;
  double tx = p.x - fx, ty = p.y - fy, tz = p.z - fz;
  tx = tx * tx * (3 - 2 * tx);
  ty = ty * ty * (3 - 2 * ty);
  tz = tz * tz * (3 - 2 * tz);
  double acc = 0;
  for (int c = 0; c < 8; ++c) {
    int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
    double w = (dx ? tx : 1 - tx) * (dy ? ty : 1 - ty) * (dz ? tz : 1 - tz);
    acc += w * hash3(ix + dx, iy + dy, iz + dz, seed);
  }
  return acc;
}

// Emits a displaced, tessellated box: each face an n x n grid of quads (12 n^2 triangles).
void emit_box(Builder &b, D3 c, D3 half, int n, double amp, uint64_t nseed, const float *m) {
  static const int axes[6][3] = {{0, 1, 2}, {0, 1, 2}, {1, 2, 0}, {1, 2, 0}, {2, 0, 1}, {2, 0, 1}};
  for (int f = 0; f < 6; ++f) {
    int na = axes[f][2], ua = axes[f][0], va = axes[f][1];
    double sgn = (f & 1) ? -1.0 : 1.0;
    auto point = [&](int i, int j) {
      double s[3];
      double h[3] = {half.x, half.y, half.z};
      s[na] = sgn * h[na];
      s[ua] = (-1.0 + 2.0 * i / n) * h[ua];
      s[va] = (-1.0 + 2.0 * j / n) * h[va];
      D3 p = {c.x + s[0], c.y + s[1], c.z + s[2]};
      double nrm[3] = {0, 0, 0};
      nrm[na] = sgn;
      double d = amp * value_noise(p * 0.35, nseed);
      return D3{p.x + nrm[0] * d, p.y + nrm[1] * d, p.z + nrm[2] * d};
    };
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        D3 p00 = point(i, j), p10 = point(i + 1, j), p01 = point(i, j + 1), p11 = point(i + 1, j + 1);
        if (sgn > 0) {
          b.tri(p00, p10, p11, m);
          b.tri(p00, p11, p01, m);
        } else {
          b.tri(p00, p11, p10, m);
          b.tri(p00, p01, p11, m);
        }
      }
  }
}

// Emits a displaced cylinder: s radial segments x h height segments plus two cap fans
// (2 s h + 2 s triangles).
void emit_cylinder(Builder &b, D3 base, double radius, double height, int s, int h, double amp,
                   uint64_t nseed, const float *m) {
  auto side = [&](int i, int j) {
    double ang = 6.283185307179586 * (i % s) / s;
    double y = height * j / h;
    D3 dir = {std::cos(ang), 0, std::sin(ang)};
    D3 p = {base.x + radius * dir.x, base.y + y, base.z + radius * dir.z};
    double d = amp * value_noise(p * 0.35, nseed);
    return D3{p.x + dir.x * d, p.y, p.z + dir.z * d};
  };
  for (int i = 0; i < s; ++i)
    for (int j = 0; j < h; ++j) {
      D3 p00 = side(i, j), p10 = side(i + 1, j), p01 = side(i, j + 1), p11 = side(i + 1, j + 1);
      b.tri(p00, p01, p11, m);
      b.tri(p00, p11, p10, m);
    }
  D3 top = {base.x, base.y + height, base.z}, bot = base;
  for (int i = 0; i < s; ++i) {
    b.tri(top, side(i + 1, h), side(i, h), m);
    b.tri(bot, side(i, 0), side(i + 1, 0), m);
  }
}

}  // namespace
}  // namespace nomad

struct nomad_scene_owned {
  nomad::Builder b;
};

using nomad::D3;

extern "C" nomad_status nomad_synth_icospheres(uint64_t seed, uint32_t instances, float extent,
                                               nomad_scene_owned **out) {
  if (!out || instances == 0 || !(extent > 0)) return NOMAD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  try {
    std::unique_ptr<nomad_scene_owned> s(new nomad_scene_owned());
    nomad::Rng r(seed);
    std::vector<D3> verts;
    std::vector<int> tris;
    nomad::icosphere(3, verts, tris);  // 20 * 4^3 = 1,280 triangles
    for (uint32_t k = 0; k < instances; ++k) {
      double rot[9];
      nomad::random_rotation(r, rot);
      double scale = r.uniform(0.5, 3.0);
      D3 tr = {r.uniform(-0.5, 0.5) * extent, r.uniform(-0.5, 0.5) * extent,
               r.uniform(-0.5, 0.5) * extent};
      float m[20];
      bool glossy = r.uniform() < 0.3;
      D3 alb = {r.uniform(0.2, 0.8), r.uniform(0.2, 0.8), r.uniform(0.2, 0.8)};
      nomad::make_material(m, alb, glossy ? D3{0.5, 0.5, 0.5} : D3{0, 0, 0}, 32.0f, {0, 0, 0}, 0.0f,
                           glossy ? (float)r.uniform(0.05, 1.0) : 1.0f);
      auto xf = [&](D3 v) {
        D3 w = {rot[0] * v.x + rot[1] * v.y + rot[2] * v.z, rot[3] * v.x + rot[4] * v.y + rot[5] * v.z,
                rot[6] * v.x + rot[7] * v.y + rot[8] * v.z};
        return w * scale + tr;
      };
      s->b.begin_object();
      for (size_t i = 0; i < tris.size(); i += 3)
        s->b.tri(xf(verts[tris[i]]), xf(verts[tris[i + 1]]), xf(verts[tris[i + 2]]), m);
      s->b.end_object();
    }
    *out = s.release();
    return NOMAD_OK;
  } catch (const std::bad_alloc &) {
    return NOMAD_ERR_OUT_OF_MEMORY;
  }
}

extern "C" nomad_status nomad_synth_city(uint64_t seed, uint32_t grid, uint32_t grid_z, float size_m,
                                         uint32_t target_tris, uint32_t median_tris,
                                         uint32_t max_tris, uint32_t emissive_quads,
                                         uint32_t emissive_tris, float emissive_sigma,
                                         nomad_scene_owned **out) {
  if (!out || grid == 0 || grid_z == 0 || !(size_m > 0) || median_tris == 0 || max_tris < 16)
    return NOMAD_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  try {
    std::unique_ptr<nomad_scene_owned> s(new nomad_scene_owned());
    nomad::Rng r(seed);
    const uint32_t cells = grid * grid_z;
    // Lognormal triangle budgets (median `median_tris`), clamped, then rescaled so the
    // total lands near `target_tris`.
    const double sigma = 1.336;
    std::vector<double> want(cells);
    double sum = 0;
    for (uint32_t c = 0; c < cells; ++c) {
      want[c] = std::min<double>(max_tris, median_tris * std::exp(sigma * r.normal()));
      sum += want[c];
    }
    double scale = target_tris > 0 ? target_tris / sum : 1.0;
    for (auto &w : want) w = std::max(16.0, std::min<double>(max_tris, w * scale));
    // Which cells carry one of the emissive quads.
    std::vector<char> lamp(cells, 0);
    for (uint32_t q = 0; q < std::min(emissive_quads, cells); ++q) {
      uint32_t c;
      do {
        c = static_cast<uint32_t>(r.next() % cells);
      } while (lamp[c]);
      lamp[c] = 1;
    }
    const double pitch = size_m / grid;
    const double half = size_m * 0.5;
    const double halfZ = pitch * grid_z * 0.5;
    uint32_t emissive_left = emissive_tris;
    for (uint32_t c = 0; c < cells; ++c) {
      uint32_t gx = c % grid, gz = c / grid;
      D3 center = {-half + (gx + 0.5) * pitch, 0.0, -halfZ + (gz + 0.5) * pitch};
      float m[20];
      bool glossy = r.uniform() < 0.35;
      D3 alb = {r.uniform(0.2, 0.8), r.uniform(0.2, 0.8), r.uniform(0.2, 0.8)};
      double spec = r.uniform(0.2, 0.9);
      nomad::make_material(m, glossy ? alb * 0.5 : alb, glossy ? D3{spec, spec, spec} : D3{0, 0, 0},
                           32.0f, {0, 0, 0}, 0.0f, glossy ? (float)r.uniform(0.05, 1.0) : 1.0f);
      float ground[20];
      nomad::make_material(ground, {0.35, 0.35, 0.33}, {0, 0, 0}, 32.0f, {0, 0, 0}, 0.0f, 1.0f);
      s->b.begin_object();
      // Ground tile of the cell.
      D3 g0 = {center.x - pitch / 2, 0, center.z - pitch / 2}, g1 = {center.x + pitch / 2, 0, center.z - pitch / 2};
      D3 g2 = {center.x + pitch / 2, 0, center.z + pitch / 2}, g3 = {center.x - pitch / 2, 0, center.z + pitch / 2};
      s->b.tri(g0, g2, g1, ground);
      s->b.tri(g0, g3, g2, ground);
      double width = r.uniform(0.25, 0.75) * pitch;
      double height = std::min(150.0, 8.0 + 25.0 * std::exp(0.8 * r.normal()));
      double amp = 0.03 * width;
      uint64_t nseed = r.next();
      int budget = static_cast<int>(want[c]) - 2;
      if (r.uniform() < 0.5) {
        int n = std::max(1, static_cast<int>(std::lround(std::sqrt(budget / 12.0))));
        D3 hb = {width / 2, height / 2, r.uniform(0.6, 1.0) * width / 2};
        nomad::emit_box(s->b, {center.x, height / 2, center.z}, hb, n, amp, nseed, m);
      } else {
        // 2 s h + 2 s triangles with h ~ s/2: s ~ sqrt(budget)
        int sseg = std::max(3, static_cast<int>(std::lround(std::sqrt(budget * 1.0))));
        int hseg = std::max(1, (budget - 2 * sseg) / (2 * sseg));
        nomad::emit_cylinder(s->b, {center.x, 0, center.z}, width / 2, height, sseg, hseg, amp, nseed, m);
      }
      if (lamp[c]) {
        float e[20];
        double power = r.uniform(5.0, 50.0);
        nomad::make_material(e, {0.8, 0.8, 0.8}, {0, 0, 0}, 32.0f, {1.0, 0.9, 0.8}, (float)power, 1.0f);
        D3 lc = {center.x + r.uniform(-0.3, 0.3) * pitch, height + r.uniform(3.0, 12.0),
                 center.z + r.uniform(-0.3, 0.3) * pitch};
        double sz = r.uniform(1.0, 4.0);
        // Facing down: u x v points to -y.
        s->b.rect(lc, {sz, 0, 0}, {0, 0, sz}, e);
      }
      // Small emissive roof triangles (ReSTIR light set), spread over the cells.
      uint32_t per = (emissive_tris + cells - 1) / cells;
      for (uint32_t k = 0; k < per && emissive_left > 0; ++k, --emissive_left) {
        float e[20];
        double power = std::exp(emissive_sigma * r.normal());
        D3 col = {r.uniform(0.6, 1.0), r.uniform(0.6, 1.0), r.uniform(0.6, 1.0)};
        nomad::make_material(e, {0.5, 0.5, 0.5}, {0, 0, 0}, 32.0f, col, (float)power, 1.0f);
        D3 p = {center.x + r.uniform(-0.5, 0.5) * width, height + 0.5 + r.uniform(0.0, 2.0),
                center.z + r.uniform(-0.5, 0.5) * width};
        double sz = r.uniform(0.3, 1.2);
        s->b.tri(p, {p.x + sz, p.y, p.z}, {p.x, p.y, p.z + sz}, e);
      }
      s->b.end_object();
    }
    *out = s.release();
    return NOMAD_OK;
  } catch (const std::bad_alloc &) {
    return NOMAD_ERR_OUT_OF_MEMORY;
  }
}

extern "C" nomad_status nomad_scene_owned_desc(const nomad_scene_owned *s, nomad_scene_desc *d) {
  if (!s || !d) return NOMAD_ERR_INVALID_ARGUMENT;
  d->prim_count = static_cast<uint32_t>(s->b.type.size());
  d->prim_type = s->b.type.data();
  d->prim_geom = s->b.geom.data();
  d->prim_material = s->b.mat.data();
  d->object_count = static_cast<uint32_t>(s->b.objFirst.size());
  d->object_first = s->b.objFirst.data();
  d->object_prims = s->b.objPrims.data();
  return NOMAD_OK;
}

extern "C" void nomad_scene_owned_free(nomad_scene_owned *s) { delete s; }
