// Scene ingest: the reference's XML scene files with OBJ/MTL meshes turned into a scene
// description (nomad_scene_load_xml).
//
// Follows SceneLoader::LoadSceneFromXML (Nomad Path Tracer/Scene/SceneLoader.cpp:344-858):
//   - the <Scene> root's settings and residency parameters (:369-687), with Scene::clear's
//     defaults (Scene/Scene.cpp:70-101);
//   - <Sphere> and <Rectangle> primitives (:694-726), a rectangle's u/v turned by Euler XYZ
//     `rotation` in degrees (rotateVectorEulerXYZ :65-84: one axis quaternion per non-zero angle,
//     applied x, then y, then z);
//   - <Mesh> (:727-825): the OBJ read once per distinct path, every vertex baked to world space
//     as position + basisX*x + basisY*y + basisZ*z (basis = scale on the diagonal unless basisX/Y/Z
//     are given, turned by `rotation`), each triangle's material chosen between the OBJ's, the
//     element's override attributes and the default fallback (:796-815), and the triangles split
//     into objects by PartitionTrianglesRecursive (:140-190): longest-axis median split with
//     std::nth_element on the centroid, until a part is within clusterMaxTriangles and
//     clusterMaxExtent;
//   - <CameraPath><Keyframe> and <ObserverCamera> (:826-855);
//   - the material attribute parsing of MaterialUtils (ParseMaterialAttributes,
//     HasOverrideAttributes, NeedsFallbackMaterial; Scene/MaterialUtils.cpp:105-289).
// Attribute numbers are read as tinyxml2 reads them (sscanf "%f", "%u"/"%x", "%llu"/"%llx",
// "%lf"; booleans as integers or true/false words), vectors with sscanf "%f,%f,%f".
//
// Differences: texture images are not decoded (every texture index is -1, as in the reference
// when an image cannot be read); a missing `position`/`u`/`v` attribute reads as 0,0,0 where the
// reference passes a null string to sscanf; the OBJ files are parsed on several threads (the
// result is the same for any thread count).
#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iterator>
#include <map>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>

#include "../../../include/nomad_scene.h"
#include "ingest.h"

namespace nomad {
namespace ingest {
namespace {

constexpr float kDegToRad = 0.0174532925199432957692f;

struct F3 {
  float x, y, z;
};
inline F3 add(F3 a, F3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline F3 mul(F3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }

// ---- tinyxml2-style attribute reads ----

bool prefix_hex(const char *p) {
  while (*p && std::isspace(static_cast<unsigned char>(*p)) && !((*p & 0xC0) == 0x80)) ++p;
  return p[0] == '0' && (p[1] == 'x' || p[1] == 'X');
}

float f_attr(const XmlElem &e, const char *n, float def) {
  const char *v = e.attr(n);
  float f;
  if (v && std::sscanf(v, "%f", &f) == 1) return f;
  return def;
}

double d_attr(const XmlElem &e, const char *n, double def) {
  const char *v = e.attr(n);
  double d;
  if (v && std::sscanf(v, "%lf", &d) == 1) return d;
  return def;
}

uint32_t u_attr(const XmlElem &e, const char *n, uint32_t def) {
  const char *v = e.attr(n);
  unsigned u;
  if (v && std::sscanf(v, prefix_hex(v) ? "%x" : "%u", &u) == 1) return u;
  return def;
}

uint64_t u64_attr(const XmlElem &e, const char *n, uint64_t def) {
  const char *v = e.attr(n);
  unsigned long long u = 0;
  if (v && std::sscanf(v, prefix_hex(v) ? "%llx" : "%llu", &u) == 1) return static_cast<uint64_t>(u);
  return def;
}

bool b_attr(const XmlElem &e, const char *n, bool def) {
  const char *v = e.attr(n);
  if (!v) return def;
  if (prefix_hex(v)) {
    unsigned u;
    if (std::sscanf(v, "%x", &u) == 1) return static_cast<int>(u) != 0;
  } else {
    int i;
    if (std::sscanf(v, "%d", &i) == 1) return i != 0;
  }
  for (const char *w : {"true", "True", "TRUE"})
    if (std::strcmp(v, w) == 0) return true;
  for (const char *w : {"false", "False", "FALSE"})
    if (std::strcmp(v, w) == 0) return false;
  return def;
}

F3 vec3(const char *s) {
  float x = 0, y = 0, z = 0;
  if (s) std::sscanf(s, "%f,%f,%f", &x, &y, &z);
  return {x, y, z};
}

// ---- rotation: q v q*, one axis quaternion per non-zero Euler angle ----

struct Quat {
  float x, y, z, w;
};

Quat qmul(const Quat &a, const Quat &b) {
  Quat o;
  o.w = a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z;
  o.x = a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y;
  o.y = a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x;
  o.z = a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w;
  return o;
}

F3 act(float angle, F3 axis, F3 v) {
  const float s = std::sin(angle * 0.5f), c = std::cos(angle * 0.5f);
  const Quat q{axis.x * s, axis.y * s, axis.z * s, c};
  const Quat p{v.x, v.y, v.z, 0.0f};
  const Quat qc{-q.x, -q.y, -q.z, q.w};
  const Quat o = qmul(qmul(q, p), qc);
  return {o.x, o.y, o.z};
}

F3 rotate_xyz(F3 v, F3 rad) {
  if (rad.x != 0.0f) v = act(rad.x, {1.0f, 0.0f, 0.0f}, v);
  if (rad.y != 0.0f) v = act(rad.y, {0.0f, 1.0f, 0.0f}, v);
  if (rad.z != 0.0f) v = act(rad.z, {0.0f, 0.0f, 1.0f}, v);
  return v;
}

// ---- materials from element attributes ----

float luminance(const float *c) { return 0.2126f * c[0] + 0.7152f * c[1] + 0.0722f * c[2]; }
float clamp01(float x) { return std::clamp(x, 0.0f, 1.0f); }

void set3(float *d, F3 v) {
  d[0] = v.x;
  d[1] = v.y;
  d[2] = v.z;
}

Mat parse_material(const XmlElem &e) {
  Mat m;
  bool hasDiffuse = false, hasSpecular = false, hasTransmission = false;
  if (const char *a = e.attr("diffuse")) {
    set3(m.diffuse(), vec3(a));
    hasDiffuse = true;
  }
  if (const char *a = e.attr("albedo")) {
    set3(m.diffuse(), vec3(a));
    hasDiffuse = true;
  }
  if (const char *a = e.attr("emission")) set3(m.emission(), vec3(a));
  m.emission_power() = f_attr(e, "emissionPower", m.emission_power());
  if (const char *a = e.attr("specular")) {
    set3(m.specular(), vec3(a));
    hasSpecular = true;
  }
  if (const char *a = e.attr("transmission")) {
    set3(m.transmission(), vec3(a));
    hasTransmission = true;
  }
  const bool hasOpacity = e.attr("opacity") != nullptr;
  m.opacity() = f_attr(e, "opacity", m.opacity());
  m.shininess() = f_attr(e, "shininess", m.shininess());
  m.roughness() = f_attr(e, "roughness", m.roughness());
  m.ior() = f_attr(e, "ior", m.ior());
  if (!hasTransmission && m.opacity() < 1.0f) {
    const float tr = 1.0f - m.opacity();
    set3(m.transmission(), {tr, tr, tr});
  }
  if (const char *a = e.attr("materialType")) {
    float type = 0.0f;
    std::sscanf(a, "%f", &type);
    if (type < 0.0f) {
      if (!hasSpecular) set3(m.specular(), {1.0f, 1.0f, 1.0f});
      m.opacity() = 1.0f;
      set3(m.transmission(), {0.0f, 0.0f, 0.0f});
      m.shininess() = std::max(m.shininess(), 256.0f);
      m.roughness() = std::min(m.roughness(), 0.02f);
    } else if (type > 0.0f) {
      if (!hasSpecular) set3(m.specular(), {1.0f, 1.0f, 1.0f});
      if (!hasTransmission) set3(m.transmission(), {1.0f, 1.0f, 1.0f});
      m.ior() = type;
      if (!hasOpacity) m.opacity() = 0.0f;
      m.shininess() = std::max(m.shininess(), 96.0f);
      m.roughness() = std::min(m.roughness(), 0.1f);
    }
  }
  m.opacity() = clamp01(m.opacity());
  m.roughness() = clamp01(m.roughness());
  m.shininess() = std::max(m.shininess(), 1.0f);
  if (!hasDiffuse && m.opacity() < 1.0f && luminance(m.diffuse()) <= 0.0f) {
    const float base = 1.0f - m.opacity();
    set3(m.diffuse(), {base, base, base});
  }
  return m;
}

bool has_override(const XmlElem &e) {
  for (const char *n : {"diffuse", "albedo", "emission", "emissionPower", "specular", "transmission", "opacity",
                        "shininess", "roughness", "ior", "materialType", "diffuseTexture", "albedoTexture",
                        "specularTexture", "normalTexture", "normalMap", "bumpTexture"})
    if (e.attr(n)) return true;
  return false;
}

bool needs_fallback(const Mat &m) {
  // no texture index is ever set here
  return luminance(m.v + 0) <= 1.0e-4f && luminance(m.v + 4) <= 1.0e-4f;
}

int strategy_of(std::string s, bool &known) {
  std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
  known = true;
  auto in = [&](std::initializer_list<const char *> l) {
    for (const char *w : l)
      if (s == w) return true;
    return false;
  };
  if (in({"energy", "importance", "energyimportance", "energy_importance"})) return 1;
  if (in({"unified", "hybrid", "unifiedscore", "unified_score"})) return 8;
  if (in({"unifiedneural", "unified_neural", "neural", "neural_unified", "neural-unified"})) return 9;
  if (in({"distance", "lod", "distance_lod", "distancelod", "distancebased"})) return 0;
  if (in({"rayhitbudget", "ray_hit_budget", "rayhits", "ray_hit", "hitbudget"})) return 2;
  if (in({"screenspacefootprint", "screen_space_footprint", "footprint", "screenspace"})) return 3;
  if (in({"probabilistic", "probability", "probabilistic_residency", "probability_residency"})) return 4;
  if (in({"alwaysresident", "always_resident", "always", "none", "off"})) return 5;
  if (in({"environment", "environmenthit", "environment_hit", "envhit", "env_hit", "env"})) return 6;
  if (in({"predictive", "predictive_environment", "predictive-env", "predictive_env"})) return 7;
  known = false;
  return 0;
}

void default_settings(nomad_scene_settings &s) {
  std::memset(&s, 0, sizeof(s));
  s.width = 1280.0f;
  s.height = 720.0f;
  s.max_ray_depth = 32;
  s.residency_strategy = 0;
  s.environment_brightness = 1.0f;
  s.texture_cap_mb = 2048.0;
  s.geometry_cap_mb = 2048.0;
  s.total_gpu_cap_mb = 4096.0;
  s.max_tile_work = 64 * 64 * 4;
  s.lod_enter_distance = 225.0f;
  s.lod_exit_distance = 275.0f;
  s.lod_enter_view_degrees = 5.0f;
  s.lod_exit_view_degrees = 12.0f;
  s.state_cooldown_frames = 5;
  s.ray_hit_cooldown_frames = 4;
  s.lod_max_toggles = 24;
  s.ray_hit_decay = 0.85f;
  s.ray_hit_target_fraction = 0.54f;
  s.ray_hit_min_active = 16;
  s.ray_hit_max_toggles = 16;
  s.screen_target_fraction = 0.68f;
  s.screen_min_pixel_coverage = 32.0f;
  s.screen_min_active = 16;
  s.screen_max_toggles = 14;
}

void read_settings(const XmlElem &r, nomad_scene_settings &s, std::string &log) {
  s.width = f_attr(r, "width", s.width);
  s.height = f_attr(r, "height", s.height);
  s.max_ray_depth = u_attr(r, "maxRayDepth", s.max_ray_depth);
  if (const char *a = r.attr("residencyStrategy")) {
    bool known = false;
    s.residency_strategy = strategy_of(a, known);
    if (!known) log += "unknown residency strategy '" + std::string(a) + "', using distance LOD\n";
  }
  s.lod_enter_distance = f_attr(r, "lodEnterDistance", s.lod_enter_distance);
  s.lod_exit_distance = f_attr(r, "lodExitDistance", s.lod_exit_distance);
  s.lod_enter_view_degrees = f_attr(r, "lodEnterViewDegrees", s.lod_enter_view_degrees);
  s.lod_exit_view_degrees = f_attr(r, "lodExitViewDegrees", s.lod_exit_view_degrees);
  s.state_cooldown_frames = u_attr(r, "residencyCooldown", s.state_cooldown_frames);
  s.lod_max_toggles = u64_attr(r, "lodToggleBudget", s.lod_max_toggles);
  s.ray_hit_decay = f_attr(r, "rayHitDecay", s.ray_hit_decay);
  s.ray_hit_target_fraction = f_attr(r, "rayHitTargetFraction", s.ray_hit_target_fraction);
  s.ray_hit_min_active = u64_attr(r, "rayHitMinActive", s.ray_hit_min_active);
  s.ray_hit_max_toggles = u64_attr(r, "rayHitToggleBudget", s.ray_hit_max_toggles);
  s.ray_hit_cooldown_frames = u_attr(r, "rayHitCooldown", s.ray_hit_cooldown_frames);
  s.ray_hit_target_memory_mb = f_attr(r, "rayHitTargetMemoryMB", s.ray_hit_target_memory_mb);
  s.screen_target_fraction = f_attr(r, "screenTargetFraction", s.screen_target_fraction);
  s.screen_min_pixel_coverage = f_attr(r, "screenMinPixelCoverage", s.screen_min_pixel_coverage);
  s.screen_min_active = u64_attr(r, "screenMinActive", s.screen_min_active);
  s.screen_max_toggles = u64_attr(r, "screenToggleBudget", s.screen_max_toggles);
  s.screen_target_memory_mb = f_attr(r, "screenTargetMemoryMB", s.screen_target_memory_mb);
  s.screen_target_memory_mb = f_attr(r, "screenspaceTargetMemoryMB", s.screen_target_memory_mb);
  s.distance_target_memory_mb = f_attr(r, "distanceTargetMemoryMB", s.distance_target_memory_mb);
  s.target_memory_mb = f_attr(r, "targetMemoryMB", s.target_memory_mb);
  s.target_resident_geometry_mb = f_attr(r, "targetResidentGeometryMB", s.target_resident_geometry_mb);
  s.start_compacted = b_attr(r, "startCompacted", s.start_compacted != 0) ? 1 : 0;
  s.texture_cap_mb = d_attr(r, "textureResidencyMemoryCapMB", s.texture_cap_mb);
  s.geometry_cap_mb = d_attr(r, "geometryResidencyMemoryCapMB", s.geometry_cap_mb);
  s.total_gpu_cap_mb = d_attr(r, "totalGpuMemoryCapMB", s.total_gpu_cap_mb);
  s.restir_enabled = b_attr(r, "restirEnabled", s.restir_enabled != 0) ? 1 : 0;
  s.environment_brightness = std::max(f_attr(r, "environmentBrightness", s.environment_brightness), 0.0f);
  uint64_t tile = u64_attr(r, "maxTileWorkPerCommand", 0);
  tile = u64_attr(r, "maxTileWork", tile);
  if (tile > 0) s.max_tile_work = std::max<uint64_t>(tile, 1);
}

// ---- the loaded scene ----

struct Tri {
  F3 v0, v1, v2;
  float uv[6];
  const Mat *mat;
};

float centroid(const Tri &t, int axis) {
  const float a = axis == 0 ? t.v0.x : axis == 1 ? t.v0.y : t.v0.z;
  const float b = axis == 0 ? t.v1.x : axis == 1 ? t.v1.y : t.v1.z;
  const float c = axis == 0 ? t.v2.x : axis == 1 ? t.v2.y : t.v2.z;
  return (a + b + c) / 3.0f;
}

void bounds(const std::vector<Tri> &tris, const std::vector<uint32_t> &idx, size_t b, size_t e, F3 &mn, F3 &mx) {
  const float big = std::numeric_limits<float>::max();
  mn = {big, big, big};
  mx = {-big, -big, -big};
  for (size_t i = b; i < e; ++i) {
    const Tri &t = tris[idx[i]];
    for (const F3 &p : {t.v0, t.v1, t.v2}) {
      mn.x = std::min(mn.x, p.x);
      mn.y = std::min(mn.y, p.y);
      mn.z = std::min(mn.z, p.z);
      mx.x = std::max(mx.x, p.x);
      mx.y = std::max(mx.y, p.y);
      mx.z = std::max(mx.z, p.z);
    }
  }
}

void partition(const std::vector<Tri> &tris, std::vector<uint32_t> &idx, size_t b, size_t e, uint64_t maxTris,
               float maxExtent, std::vector<std::pair<size_t, size_t>> &parts) {
  const size_t count = e - b;
  if (count == 0) return;
  F3 mn, mx;
  bounds(tris, idx, b, e, mn, mx);
  const F3 ext{mx.x - mn.x, mx.y - mn.y, mx.z - mn.z};
  float longest = ext.x;
  int axis = 0;
  if (ext.y > longest) {
    longest = ext.y;
    axis = 1;
  }
  if (ext.z > longest) {
    longest = ext.z;
    axis = 2;
  }
  const bool triOk = maxTris == 0 || count <= maxTris;
  const bool extOk = maxExtent <= 0.0f || longest <= maxExtent;
  if ((triOk && extOk) || count <= 1) {
    parts.emplace_back(b, e);
    return;
  }
  const size_t mid = b + count / 2;
  if (mid == b || mid == e) {
    parts.emplace_back(b, e);
    return;
  }
  // Same comparisons and exchanges as the reference's nth_element over its primitive array.
  std::nth_element(idx.begin() + static_cast<std::ptrdiff_t>(b), idx.begin() + static_cast<std::ptrdiff_t>(mid),
                   idx.begin() + static_cast<std::ptrdiff_t>(e), [&](uint32_t x, uint32_t y) {
                     return centroid(tris[x], axis) < centroid(tris[y], axis);
                   });
  partition(tris, idx, b, mid, maxTris, maxExtent, parts);
  partition(tris, idx, mid, e, maxTris, maxExtent, parts);
}

}  // namespace
}  // namespace ingest
}  // namespace nomad

struct nomad_loaded_scene {
  std::vector<int32_t> type;
  std::vector<float> geom, mat;
  std::vector<uint32_t> first, count;
  std::vector<int32_t> group;
  nomad_scene_settings settings;
  std::vector<nomad_camera_keyframe> keys;
  nomad_observer_camera observer;
  int32_t hasObserver = 0;
  std::string env, log;
  uint32_t meshFiles = 0, meshFailed = 0;
};

namespace {

using namespace nomad::ingest;
namespace fs = std::filesystem;

void put(float *d, F3 v) {
  d[0] = v.x;
  d[1] = v.y;
  d[2] = v.z;
}

void load(const std::string &path, uint32_t threads, nomad_loaded_scene &S) {
  std::string text;
  {
    std::ifstream f(path.c_str(), std::ios::binary);
    if (!f) throw std::invalid_argument("cannot read scene XML " + path);
    text.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  }
  std::vector<XmlElem> roots;
  std::string err;
  if (!parse_xml(text, roots, err)) throw std::invalid_argument("scene XML " + path + ": " + err);
  const XmlElem *root = nullptr;
  for (const XmlElem &e : roots)
    if (e.name == "Scene") {
      root = &e;
      break;
    }
  if (!root) throw std::invalid_argument("scene XML " + path + " has no <Scene> root");
  const fs::path baseDir = fs::path(path).parent_path();

  default_settings(S.settings);
  read_settings(*root, S.settings, S.log);
  if (const char *a = root->attr("environmentTexture"); a && a[0]) {
    fs::path p(a);
    if (p.is_relative()) p = baseDir / p;
    S.env = p.lexically_normal().string();
  }

  // Distinct mesh files in order of first use, parsed in parallel.
  std::vector<std::string> files;
  std::unordered_map<std::string, size_t> fileIndex;
  auto mesh_path = [&](const XmlElem &e) {
    const char *f = e.attr("file");
    return (baseDir / (f ? f : "")).lexically_normal().string();
  };
  for (const XmlElem &e : root->children)
    if (e.name == "Mesh") {
      const std::string p = mesh_path(e);
      if (fileIndex.emplace(p, files.size()).second) files.push_back(p);
    }
  std::vector<Mesh> meshes(files.size());
  {
    unsigned nt = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    nt = static_cast<unsigned>(std::min<size_t>(nt, files.size()));
    std::atomic<size_t> next{0};
    std::exception_ptr failure;
    std::mutex failureLock;
    auto work = [&]() {
      try {
        for (size_t i; (i = next.fetch_add(1)) < files.size();) {
          const fs::path p(files[i]);
          std::string dir;
          if (p.has_parent_path()) {
            dir = p.parent_path().string();
            if (!dir.empty() && dir.back() != fs::path::preferred_separator)
              dir.push_back(fs::path::preferred_separator);
          }
          load_obj(files[i], dir, meshes[i]);
        }
      } catch (...) {  // handed to the calling thread, which turns it into a status
        std::lock_guard<std::mutex> g(failureLock);
        if (!failure) failure = std::current_exception();
        next.store(files.size());
      }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    if (failure) std::rethrow_exception(failure);
  }
  S.meshFiles = static_cast<uint32_t>(files.size());
  for (size_t i = 0; i < files.size(); ++i) {
    if (!meshes[i].ok) {
      ++S.meshFailed;
      S.log += "failed to load OBJ " + files[i] + ": " + meshes[i].message + "\n";
    } else if (meshes[i].invalidTris) {
      S.log += "OBJ " + files[i] + ": " + std::to_string(meshes[i].invalidTris) +
               " triangles with out-of-range vertex indices dropped\n";
    }
  }

  // Every <Sphere>, <Rectangle> and <Mesh> owns a known range of primitives (a mesh's split into
  // objects only permutes inside its range), so the output is sized first, the elements are baked
  // and split on the worker threads into their own ranges, and the object lists are joined in
  // element order: the same arrays for any thread count.
  struct Part {
    const XmlElem *e;
    int kind;  // NOMAD_PRIM_SPHERE / NOMAD_PRIM_RECTANGLE, or -1 for a mesh
    size_t mesh;
    int group;
    size_t base, count;
    std::vector<std::pair<size_t, size_t>> objs;  // (first, count) relative to base
  };
  std::vector<Part> parts;
  size_t total = 0;
  int nextGroup = 0;
  for (const XmlElem &e : root->children) {
    if (e.name == "Sphere" || e.name == "Rectangle") {
      parts.push_back({&e, e.name == "Sphere" ? NOMAD_PRIM_SPHERE : NOMAD_PRIM_RECTANGLE, 0, -1, total, 1, {}});
      total += 1;
    } else if (e.name == "Mesh") {
      const size_t m = fileIndex.at(mesh_path(e));
      const size_t nt = meshes[m].triMat.size();
      parts.push_back({&e, -1, m, nextGroup++, total, nt, {}});
      total += nt;
    } else if (e.name == "CameraPath") {
      for (const XmlElem &k : e.children) {
        if (k.name != "Keyframe") continue;
        nomad_camera_keyframe K{};
        K.frame = u_attr(k, "frame", 0);
        put(K.position, vec3(k.attr("position")));
        put(K.look_at, vec3(k.attr("lookAt")));
        const char *up = k.attr("up");
        put(K.up, up ? vec3(up) : F3{0.0f, 1.0f, 0.0f});
        K.aperture = f_attr(k, "aperture", 0.0f);
        K.focus_distance = f_attr(k, "focusDistance", 1.0f);
        S.keys.push_back(K);
      }
    } else if (e.name == "ObserverCamera") {
      nomad_observer_camera &o = S.observer;
      if (const char *a = e.attr("position")) put(o.position, vec3(a));
      if (const char *a = e.attr("lookAt")) put(o.look_at, vec3(a));
      if (const char *a = e.attr("up")) put(o.up, vec3(a));
      o.vertical_fov = f_attr(e, "verticalFov", o.vertical_fov);
      o.aperture = f_attr(e, "aperture", o.aperture);
      o.focus_distance = f_attr(e, "focusDistance", o.focus_distance);
      S.hasObserver = 1;
    }
  }
  S.type.resize(total);
  S.geom.resize(total * 15);
  S.mat.resize(total * 20);

  const Mat fallback;
  auto emit = [&](Part &P, std::vector<Tri> &tris, std::vector<uint32_t> &idx) {
    const XmlElem &e = *P.e;
    int32_t *type = S.type.data() + P.base;
    float *geom = S.geom.data() + 15 * P.base;
    float *mat = S.mat.data() + 20 * P.base;
    if (P.kind == NOMAD_PRIM_SPHERE) {
      std::memset(geom, 0, 15 * sizeof(float));
      put(geom, vec3(e.attr("position")));
      geom[3] = f_attr(e, "radius", 1.0f);
      std::memcpy(mat, parse_material(e).v, 20 * sizeof(float));
      type[0] = NOMAD_PRIM_SPHERE;
      P.objs.emplace_back(0, 1);
      return;
    }
    if (P.kind == NOMAD_PRIM_RECTANGLE) {
      F3 c = vec3(e.attr("position")), u = vec3(e.attr("u")), v = vec3(e.attr("v"));
      if (const char *r = e.attr("rotation")) {
        const F3 rad = mul(vec3(r), kDegToRad);
        u = rotate_xyz(u, rad);
        v = rotate_xyz(v, rad);
      }
      std::memset(geom, 0, 15 * sizeof(float));
      put(geom, c);
      put(geom + 3, u);
      put(geom + 6, v);
      std::memcpy(mat, parse_material(e).v, 20 * sizeof(float));
      type[0] = NOMAD_PRIM_RECTANGLE;
      P.objs.emplace_back(0, 1);
      return;
    }
    const Mesh &mesh = meshes[P.mesh];
    const F3 pos = vec3(e.attr("position"));
    const float scale = f_attr(e, "scale", 1.0f);
    F3 bx{scale, 0.0f, 0.0f}, by{0.0f, scale, 0.0f}, bz{0.0f, 0.0f, scale};
    F3 rotDeg{0.0f, 0.0f, 0.0f};
    if (const char *a = e.attr("rotation")) rotDeg = vec3(a);
    if (const char *a = e.attr("basisX")) bx = vec3(a);
    if (const char *a = e.attr("basisY")) by = vec3(a);
    if (const char *a = e.attr("basisZ")) bz = vec3(a);
    if (rotDeg.x != 0.0f || rotDeg.y != 0.0f || rotDeg.z != 0.0f) {
      const F3 rad = mul(rotDeg, kDegToRad);
      bx = rotate_xyz(bx, rad);
      by = rotate_xyz(by, rad);
      bz = rotate_xyz(bz, rad);
    }
    const Mat over = parse_material(e);
    const bool explicitOver = has_override(e);
    const uint64_t maxTris = u64_attr(e, "clusterMaxTriangles", 0);
    const float maxExtent = f_attr(e, "clusterMaxExtent", 0.0f);
    auto bake = [&](uint32_t vi) {
      const float *p = &mesh.vertices[3 * static_cast<size_t>(vi)];
      return add(add(add(pos, mul(bx, p[0])), mul(by, p[1])), mul(bz, p[2]));
    };
    const size_t nt = P.count;
    if (nt == 0) return;
    tris.resize(nt);
    for (size_t t = 0; t < nt; ++t) {
      Tri &T = tris[t];
      T.v0 = bake(mesh.tris[3 * t]);
      T.v1 = bake(mesh.tris[3 * t + 1]);
      T.v2 = bake(mesh.tris[3 * t + 2]);
      std::memcpy(T.uv, &mesh.uvs[6 * t], sizeof(T.uv));
      const Mat *chosen = &over;
      bool usingOver = true;
      const int mid = mesh.triMat[t];
      if (mid >= 0 && static_cast<size_t>(mid) < mesh.materials.size()) {
        chosen = &mesh.materials[mid];
        usingOver = false;
      }
      const bool allowFallback = !(usingOver && explicitOver);
      if (allowFallback && (mid < 0 || needs_fallback(*chosen))) chosen = &fallback;
      T.mat = chosen;
    }
    idx.resize(nt);
    for (size_t t = 0; t < nt; ++t) idx[t] = static_cast<uint32_t>(t);
    if ((maxTris == 0 && maxExtent <= 0.0f) || nt <= 1)
      P.objs.emplace_back(0, nt);
    else
      partition(tris, idx, 0, nt, maxTris, maxExtent, P.objs);
    for (size_t k = 0; k < nt; ++k) {
      const Tri &T = tris[idx[k]];
      float *g = geom + 15 * k;
      put(g, T.v0);
      put(g + 3, T.v1);
      put(g + 6, T.v2);
      std::memcpy(g + 9, T.uv, sizeof(T.uv));
      std::memcpy(mat + 20 * k, T.mat->v, 20 * sizeof(float));
      type[k] = NOMAD_PRIM_TRIANGLE;
    }
    // partition() reports [begin, end) pairs; keep (first, count)
    for (auto &o : P.objs) o.second -= o.first;
  };
  {
    unsigned nt = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    nt = static_cast<unsigned>(std::max<size_t>(1, std::min<size_t>(nt, parts.size())));
    std::atomic<size_t> next{0};
    std::exception_ptr failure;
    std::mutex failureLock;
    auto work = [&]() {
      std::vector<Tri> tris;
      std::vector<uint32_t> idx;
      try {
        for (size_t i; (i = next.fetch_add(1)) < parts.size();) emit(parts[i], tris, idx);
      } catch (...) {
        std::lock_guard<std::mutex> g(failureLock);
        if (!failure) failure = std::current_exception();
        next.store(parts.size());
      }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < nt; ++t) pool.emplace_back(work);
    work();
    for (auto &t : pool) t.join();
    if (failure) std::rethrow_exception(failure);
  }
  for (const Part &P : parts)
    for (const auto &o : P.objs) {
      S.first.push_back(static_cast<uint32_t>(P.base + o.first));
      S.count.push_back(static_cast<uint32_t>(o.second));
      S.group.push_back(P.group);
    }
}

void default_observer(nomad_observer_camera &o) {
  std::memset(&o, 0, sizeof(o));
  o.look_at[2] = -1.0f;
  o.up[1] = 1.0f;
  o.vertical_fov = 60.0f;
  o.focus_distance = 1.0f;
}

}  // namespace

namespace {
thread_local std::string tLastError;
}

extern "C" const char *nomad_scene_last_error(void) { return tLastError.c_str(); }

extern "C" nomad_status nomad_scene_load_xml(const char *path, uint32_t threads, nomad_loaded_scene **out) {
  tLastError.clear();
  if (!path || !out) {
    tLastError = "path and out must not be null";
    return NOMAD_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  try {
    std::unique_ptr<nomad_loaded_scene> s(new nomad_loaded_scene());
    default_observer(s->observer);
    load(path, threads, *s);
    *out = s.release();
    return NOMAD_OK;
  } catch (const std::bad_alloc &) {
    tLastError = "out of host memory";
    return NOMAD_ERR_OUT_OF_MEMORY;
  } catch (const std::exception &e) {
    tLastError = e.what();
    return NOMAD_ERR_INVALID_ARGUMENT;
  }
}

extern "C" nomad_status nomad_loaded_scene_view_get(const nomad_loaded_scene *s, nomad_loaded_scene_view *v) {
  if (!s || !v) return NOMAD_ERR_INVALID_ARGUMENT;
  std::memset(v, 0, sizeof(*v));
  v->scene.prim_count = static_cast<uint32_t>(s->type.size());
  v->scene.prim_type = s->type.data();
  v->scene.prim_geom = s->geom.data();
  v->scene.prim_material = s->mat.data();
  v->scene.object_count = static_cast<uint32_t>(s->first.size());
  v->scene.object_first = s->first.data();
  v->scene.object_prims = s->count.data();
  v->object_mesh_group = s->group.data();
  v->settings = s->settings;
  v->keyframe_count = static_cast<uint32_t>(s->keys.size());
  v->has_observer = s->hasObserver;
  v->keyframes = s->keys.data();
  v->observer = s->observer;
  v->environment_texture = s->env.c_str();
  v->mesh_files = s->meshFiles;
  v->mesh_files_failed = s->meshFailed;
  v->log = s->log.c_str();
  return NOMAD_OK;
}

extern "C" void nomad_loaded_scene_free(nomad_loaded_scene *s) { delete s; }
