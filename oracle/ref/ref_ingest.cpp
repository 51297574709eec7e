// ORACLE glue — test infrastructure only. Runs the reference's own scene loader
// (SceneLoader::LoadSceneFromXML with its MaterialUtils, the vendored tinyxml2 and
// tinyobjloader, all compiled here from the reference sources) and hands back what it put into
// the Scene: primitives (type, geometry, material) in load order, objects with their mesh
// groups, the root's settings, the camera path and the observer camera. Used to generate the
// golden fixtures of the ingest tests and to check whole reference scenes.
//
// Texture images are not decoded here (texture residency is outside the checked path): the
// stand-in LoadTextureImage below fails, so every texture index is -1, exactly as the
// reference behaves when a texture file cannot be read.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/nomad_scene.h"
#include "Scene.h"
#include "SceneLoader.h"
#include "TextureLoader.h"

namespace NomadPathTracer {
TextureColorSpace DetermineTextureColorSpace(const std::string &, TextureUsage) {
  return TextureColorSpace::sRGB;
}
bool LoadTextureImage(const std::string &, LoadedTextureImage &, TextureUsage) { return false; }
}  // namespace NomadPathTracer

using namespace NomadPathTracer;

namespace {
struct RefLoaded {
  std::vector<int32_t> type;
  std::vector<float> geom, mat;
  std::vector<uint32_t> first, count;
  std::vector<int32_t> group;
  nomad_scene_settings settings{};
  std::vector<nomad_camera_keyframe> keys;
  nomad_observer_camera observer{};
  int32_t hasObserver = 0;
  std::string env;
};

void put3(float *d, const simd::float3 &v) {
  d[0] = v.x;
  d[1] = v.y;
  d[2] = v.z;
}
}  // namespace

extern "C" int ref_load_xml(const char *path, void **out) {
  if (!path || !out) return 2;
  Scene *scene = new Scene();
  scene->clear();
  const bool ok = SceneLoader::LoadSceneFromXML(path, scene);
  if (!ok) {
    delete scene;
    *out = nullptr;
    return 1;
  }
  RefLoaded *r = new RefLoaded();
  const auto &prims = scene->getPrimitives();
  for (const Primitive &p : prims) {
    r->type.push_back(static_cast<int32_t>(p.type));
    float g[15] = {0};
    if (p.type == PrimitiveType::Sphere) {
      put3(g, p.sphere.center);
      g[3] = p.sphere.radius;
    } else if (p.type == PrimitiveType::Rectangle) {
      put3(g, p.rectangle.center);
      put3(g + 3, p.rectangle.u);
      put3(g + 6, p.rectangle.v);
    } else {
      put3(g, p.triangle.v0);
      put3(g + 3, p.triangle.v1);
      put3(g + 6, p.triangle.v2);
      g[9] = p.triangle.uv0.x;
      g[10] = p.triangle.uv0.y;
      g[11] = p.triangle.uv1.x;
      g[12] = p.triangle.uv1.y;
      g[13] = p.triangle.uv2.x;
      g[14] = p.triangle.uv2.y;
    }
    r->geom.insert(r->geom.end(), g, g + 15);
    const auto enc = encodeMaterial(p.material);
    for (const auto &f4 : enc) r->mat.insert(r->mat.end(), {f4.x, f4.y, f4.z, f4.w});
  }
  for (const auto &o : scene->getObjects()) {
    r->first.push_back(static_cast<uint32_t>(o.firstPrimitive));
    r->count.push_back(static_cast<uint32_t>(o.primitiveCount));
    r->group.push_back(o.meshGroupId);
  }
  nomad_scene_settings &s = r->settings;
  s.width = scene->screenSize.x;
  s.height = scene->screenSize.y;
  s.max_ray_depth = scene->maxRayDepth;
  s.residency_strategy = static_cast<int32_t>(scene->getResidencyStrategy());
  s.start_compacted = scene->getStartCompacted() ? 1 : 0;
  s.restir_enabled = scene->getRestirEnabled() ? 1 : 0;
  s.environment_brightness = scene->getEnvironmentBrightness();
  s.texture_cap_mb = scene->getTextureResidencyMemoryCapMB();
  s.geometry_cap_mb = scene->getGeometryResidencyMemoryCapMB();
  s.total_gpu_cap_mb = scene->getTotalGpuMemoryCapMB();
  s.max_tile_work = static_cast<uint64_t>(scene->getMaxTileSampleWorkPerCommand());
  const ResidencyParameters &p = scene->getResidencyParameters();
  s.lod_enter_distance = p.lodEnterDistance;
  s.lod_exit_distance = p.lodExitDistance;
  s.lod_enter_view_degrees = p.lodEnterViewDegrees;
  s.lod_exit_view_degrees = p.lodExitViewDegrees;
  s.state_cooldown_frames = p.stateCooldownFrames;
  s.ray_hit_cooldown_frames = p.rayHitRebuildCooldownFrames;
  s.lod_max_toggles = p.lodMaxTogglesPerFrame;
  s.ray_hit_decay = p.rayHitDecay;
  s.ray_hit_target_fraction = p.rayHitTargetFraction;
  s.ray_hit_min_active = p.rayHitMinActivePrimitives;
  s.ray_hit_max_toggles = p.rayHitMaxTogglesPerFrame;
  s.screen_target_fraction = p.screenFootprintTargetFraction;
  s.screen_min_pixel_coverage = p.screenFootprintMinPixelCoverage;
  s.screen_min_active = p.screenFootprintMinActivePrimitives;
  s.screen_max_toggles = p.screenFootprintMaxTogglesPerFrame;
  s.ray_hit_target_memory_mb = p.rayHitTargetMemoryMB;
  s.screen_target_memory_mb = p.screenTargetMemoryMB;
  s.distance_target_memory_mb = p.distanceTargetMemoryMB;
  s.target_memory_mb = p.targetMemoryMB;
  s.target_resident_geometry_mb = p.targetResidentGeometryMB;
  for (const CameraKeyframe &k : scene->cameraPath) {
    nomad_camera_keyframe o{};
    o.frame = k.frame;
    put3(o.position, k.position);
    put3(o.look_at, k.lookAt);
    put3(o.up, k.up);
    o.aperture = k.aperture;
    o.focus_distance = k.focusDistance;
    r->keys.push_back(o);
  }
  if (scene->hasObserverCamera()) {
    const ObserverCamera &c = scene->getObserverCamera();
    r->hasObserver = 1;
    put3(r->observer.position, c.position);
    put3(r->observer.look_at, c.lookAt);
    put3(r->observer.up, c.up);
    r->observer.vertical_fov = c.verticalFov;
    r->observer.aperture = c.aperture;
    r->observer.focus_distance = c.focusDistance;
  }
  r->env = scene->getEnvironmentTexturePath();
  delete scene;
  *out = r;
  return 0;
}

// counts: [0] primitives, [1] objects, [2] keyframes, [3] has observer
extern "C" void ref_loaded_counts(void *h, uint32_t *out) {
  const RefLoaded *r = static_cast<const RefLoaded *>(h);
  out[0] = static_cast<uint32_t>(r->type.size());
  out[1] = static_cast<uint32_t>(r->first.size());
  out[2] = static_cast<uint32_t>(r->keys.size());
  out[3] = static_cast<uint32_t>(r->hasObserver);
}

extern "C" void ref_loaded_arrays(void *h, int32_t *type, float *geom, float *mat, uint32_t *first,
                                  uint32_t *count, int32_t *group, nomad_scene_settings *settings,
                                  nomad_camera_keyframe *keys, nomad_observer_camera *observer,
                                  char *env, uint32_t envCap) {
  const RefLoaded *r = static_cast<const RefLoaded *>(h);
  std::memcpy(type, r->type.data(), r->type.size() * 4);
  std::memcpy(geom, r->geom.data(), r->geom.size() * 4);
  std::memcpy(mat, r->mat.data(), r->mat.size() * 4);
  std::memcpy(first, r->first.data(), r->first.size() * 4);
  std::memcpy(count, r->count.data(), r->count.size() * 4);
  std::memcpy(group, r->group.data(), r->group.size() * 4);
  *settings = r->settings;
  if (!r->keys.empty()) std::memcpy(keys, r->keys.data(), r->keys.size() * sizeof(nomad_camera_keyframe));
  *observer = r->observer;
  if (envCap) {
    std::strncpy(env, r->env.c_str(), envCap - 1);
    env[envCap - 1] = 0;
  }
}

extern "C" void ref_loaded_free(void *h) { delete static_cast<RefLoaded *>(h); }
