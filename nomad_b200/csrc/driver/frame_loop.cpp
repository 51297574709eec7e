// nomad_frame_loop: a C++ frame loop over libnomad_rt, the stand-in for the reference's
// Renderer::draw (Nomad Path Tracer/Renderer/Renderer.cpp:7317-7581) with its per-frame
// residency update (updateResidency, RendererResidency.cpp:165-287) and the hit-counter readback
// that feeds it (processRayHitCounters, Renderer.cpp:8004-8522).
//
// Per frame: move the camera along a seeded orbit (or along the scene file's camera path), render
// the view (one batched call that replays a captured CUDA graph after the first frame), read the
// radiance back to the host, then run one device residency step under the chosen policy and byte
// budget. Prints one JSON line; optionally writes the last frame as a PFM image (little-endian,
// bottom row first).
//
// --scene xml:FILE loads one of the reference's scene files (nomad_scene_load_xml); its
// <CameraPath> keyframes, interpolated by frame number as the reference does, replace the orbit, and its
// width, height and maxRayDepth apply unless given on the command line.
//
//   nomad_frame_loop [--scene city|icospheres|xml:FILE] [--width W] [--height H] [--spp S] [--depth D]
//                    [--frames F] [--policy always|rayhit|learned] [--budget FRACTION]
//                    [--mlp WEIGHTS] [--seed N] [--out FILE.pfm]
//
// --mlp reads a model file (nomad_mlp_save) or a raw parameter blob (NOMAD_MLP_PARAMS float32
// values, as nomad_mlp_get writes it); the learned policy needs one.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../../include/nomad_rt.h"

namespace {

struct Args {
  std::string scene = "city", policy = "always", out, mlp;
  uint32_t width = 640, height = 360, spp = 2, depth = 2, frames = 8, seed = 17;
  float budget = 0.4f;
  bool widthSet = false, heightSet = false, depthSet = false;
};

bool parse(int argc, char **argv, Args &a) {
  for (int i = 1; i < argc; ++i) {
    std::string k = argv[i];
    auto next = [&](const char *what) -> const char * {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value for %s\n", what);
        std::exit(2);
      }
      return argv[++i];
    };
    if (k == "--scene") a.scene = next("--scene");
    else if (k == "--policy") a.policy = next("--policy");
    else if (k == "--out") a.out = next("--out");
    else if (k == "--mlp") a.mlp = next("--mlp");
    else if (k == "--width") a.width = (uint32_t)std::atoi(next("--width")), a.widthSet = true;
    else if (k == "--height") a.height = (uint32_t)std::atoi(next("--height")), a.heightSet = true;
    else if (k == "--spp") a.spp = (uint32_t)std::atoi(next("--spp"));
    else if (k == "--depth") a.depth = (uint32_t)std::atoi(next("--depth")), a.depthSet = true;
    else if (k == "--frames") a.frames = (uint32_t)std::atoi(next("--frames"));
    else if (k == "--seed") a.seed = (uint32_t)std::atoi(next("--seed"));
    else if (k == "--budget") a.budget = (float)std::atof(next("--budget"));
    else {
      std::fprintf(stderr, "unknown argument %s\n", k.c_str());
      return false;
    }
  }
  return true;
}

#define CHECK(call)                                                                             \
  do {                                                                                          \
    nomad_status st_ = (call);                                                                  \
    if (st_ != NOMAD_OK) {                                                                      \
      std::fprintf(stderr, "%s failed (%d): %s\n", #call, (int)st_, ctx ? nomad_last_error(ctx) : ""); \
      return 1;                                                                                 \
    }                                                                                           \
  } while (0)

// Camera of frame f: an orbit around the scene centre at a fixed height, looking at the centre.
void orbit(const float bmin[3], const float bmax[3], uint32_t f, float pos[3], float look[3]) {
  const float cx = 0.5f * (bmin[0] + bmax[0]), cz = 0.5f * (bmin[2] + bmax[2]);
  const float ex = bmax[0] - bmin[0], ez = bmax[2] - bmin[2];
  const float r = 0.45f * std::sqrt(ex * ex + ez * ez);
  const float ang = 0.05f * (float)f;
  pos[0] = cx + r * std::cos(ang);
  pos[1] = bmin[1] + 0.25f * (bmax[1] - bmin[1]) + 0.08f * r;
  pos[2] = cz + r * std::sin(ang);
  look[0] = cx;
  look[1] = bmin[1];
  look[2] = cz;
}

// Camera of frame f on a keyframed path, as Renderer::updateCameraStates interpolates it
// (Renderer.cpp:6826-6880): the first keyframe up to its frame, the last one from its frame on,
// otherwise linear on the first segment with k0.frame <= f <= k1.frame.
void along_path(const nomad_camera_keyframe *k, uint32_t n, uint32_t f, float pos[3], float look[3], float up[3]) {
  const nomad_camera_keyframe *a = &k[0], *b = &k[0];
  float t = 0.0f;
  if (f <= k[0].frame) {
    a = b = &k[0];
  } else if (f >= k[n - 1].frame) {
    a = b = &k[n - 1];
  } else {
    for (uint32_t i = 0; i + 1 < n; ++i)
      if (f >= k[i].frame && f <= k[i + 1].frame) {
        a = &k[i];
        b = &k[i + 1];
        // two keyframes on one frame: the earlier one (the reference divides 0 by 0 there)
        t = b->frame > a->frame ? (float)(f - a->frame) / (float)(b->frame - a->frame) : 0.0f;
        break;
      }
  }
  for (int c = 0; c < 3; ++c) {
    pos[c] = a->position[c] + t * (b->position[c] - a->position[c]);
    look[c] = a->look_at[c] + t * (b->look_at[c] - a->look_at[c]);
    up[c] = a->up[c] + t * (b->up[c] - a->up[c]);
  }
}

}  // namespace

int main(int argc, char **argv) {
  Args a;
  if (!parse(argc, argv, a)) return 2;
  nomad_ctx *ctx = nullptr;
  nomad_scene_owned *scene = nullptr;
  nomad_loaded_scene *loaded = nullptr;
  nomad_loaded_scene_view lv;
  std::memset(&lv, 0, sizeof(lv));
  nomad_scene_desc desc;
  if (a.scene == "city") {
    CHECK(nomad_synth_city(a.seed, 32, 32, 1000.0f, 600000, 1000, 50000, 32, 0, 1.5f, &scene));
  } else if (a.scene == "icospheres") {
    CHECK(nomad_synth_icospheres(a.seed, 64, 100.0f, &scene));
  } else if (a.scene.rfind("xml:", 0) == 0) {
    CHECK(nomad_scene_load_xml(a.scene.c_str() + 4, 0, &loaded));
    CHECK(nomad_loaded_scene_view_get(loaded, &lv));
    if (lv.scene.prim_count == 0) {
      std::fprintf(stderr, "%s holds no primitives\n", a.scene.c_str() + 4);
      return 2;
    }
    if (!a.widthSet) a.width = (uint32_t)lv.settings.width;
    if (!a.heightSet) a.height = (uint32_t)lv.settings.height;
    if (!a.depthSet) a.depth = lv.settings.max_ray_depth;
  } else {
    std::fprintf(stderr, "unknown scene %s\n", a.scene.c_str());
    return 2;
  }
  if (loaded)
    desc = lv.scene;
  else
    CHECK(nomad_scene_owned_desc(scene, &desc));
  nomad_scenebvh *bvh = nullptr;
  CHECK(nomad_scenebvh_build(&desc, 0, &bvh));
  nomad_scenebvh_view v;
  CHECK(nomad_scenebvh_view_get(bvh, &v));
  nomad_config cfg{0, 0};
  CHECK(nomad_create(&cfg, &ctx));
  CHECK(nomad_scene_upload(ctx, v.bvh_nodes, v.bvh_node_count, v.tlas_nodes, v.tlas_node_count, v.prims,
                           v.materials, v.prim_indices, v.prim_count, v.instances, v.object_count));
  // scene bounds from the object boxes
  float bmin[3] = {INFINITY, INFINITY, INFINITY}, bmax[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint32_t o = 0; o < v.object_count; ++o)
    for (int k = 0; k < 3; ++k) {
      bmin[k] = std::fmin(bmin[k], v.object_bounds[6 * o + k]);
      bmax[k] = std::fmax(bmax[k], v.object_bounds[6 * o + 3 + k]);
    }
  std::vector<uint64_t> bytes(v.object_count);
  CHECK(nomad_object_bytes(ctx, bytes.data()));
  uint64_t total = 0;
  for (uint64_t b : bytes) total += b;

  nomad_residency_params prm;
  std::memset(&prm, 0, sizeof(prm));
  prm.policy = NOMAD_POLICY_ALWAYS;
  if (a.policy == "rayhit") prm.policy = NOMAD_POLICY_RAYHIT_BUDGET;
  else if (a.policy == "learned") prm.policy = NOMAD_POLICY_LEARNED;
  else if (a.policy != "always") {
    std::fprintf(stderr, "unknown policy %s\n", a.policy.c_str());
    return 2;
  }
  prm.budget_bytes = prm.policy == NOMAD_POLICY_ALWAYS ? 0 : (uint64_t)((double)a.budget * (double)total);
  prm.hit_decay = 0.85f;
  prm.camera_motion = 0.3f;
  prm.memory_pressure = 0.0f;
  prm.reserve_base = 0.02f;
  prm.reserve_motion = 0.06f;
  // hit-probability posterior with the reference's defaults (ResidencyParameters, Scene.h:90-100)
  prm.probability_decay = 0.9f;
  prm.probability_window = 64.0f;
  prm.probability_idle_decay = 0.9f;
  prm.probability_threshold = 0.5f;
  if (prm.policy == NOMAD_POLICY_LEARNED) {
    if (a.mlp.empty()) {
      std::fprintf(stderr, "the learned policy needs --mlp WEIGHTS\n");
      return 2;
    }
    char magic[4] = {0, 0, 0, 0};
    FILE *f = std::fopen(a.mlp.c_str(), "rb");
    if (!f || std::fread(magic, 1, 4, f) != 4) {
      std::fprintf(stderr, "cannot read %s\n", a.mlp.c_str());
      if (f) std::fclose(f);
      return 2;
    }
    if (std::memcmp(magic, "NMLP", 4) == 0) {  // a model file written by nomad_mlp_save
      std::fclose(f);
      CHECK(nomad_mlp_load(ctx, a.mlp.c_str()));
    } else {  // a raw parameter blob
      std::vector<float> blob(NOMAD_MLP_PARAMS);
      std::rewind(f);
      const bool ok = std::fread(blob.data(), 4, blob.size(), f) == blob.size();
      std::fclose(f);
      if (!ok) {
        std::fprintf(stderr, "cannot read %s\n", a.mlp.c_str());
        return 2;
      }
      CHECK(nomad_mlp_init(ctx, 1));
      CHECK(nomad_mlp_set(ctx, blob.data()));
    }
  }

  const size_t pixels = (size_t)a.width * a.height;
  std::vector<float> radiance(pixels * 3);
  double render_ms = 0.0, step_ms = 0.0;
  nomad_view view;
  CHECK(nomad_reset_render_stats(ctx));
  for (uint32_t f = 0; f < a.frames; ++f) {
    float pos[3], look[3], up[3] = {0.0f, 1.0f, 0.0f};
    if (loaded && lv.keyframe_count)
      along_path(lv.keyframes, lv.keyframe_count, f, pos, look, up);
    else
      orbit(bmin, bmax, f, pos, look);
    CHECK(nomad_view_pinhole(pos, look, up, 60.0f, a.width, a.height, &view));
    view.spp = a.spp;
    view.max_depth = a.depth;
    view.seed_lo = a.seed;
    view.frame = f;
    auto t0 = std::chrono::steady_clock::now();
    CHECK(nomad_render_frame(ctx, &view, 1, radiance.data(), NOMAD_TRACE_COUNT_HITS));
    auto t1 = std::chrono::steady_clock::now();
    CHECK(nomad_residency_step(ctx, &prm, &view, nullptr));
    CHECK(nomad_sync(ctx));
    auto t2 = std::chrono::steady_clock::now();
    if (f > 0) {  // the first frame captures the frame graph
      render_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
      step_ms += std::chrono::duration<double, std::milli>(t2 - t1).count();
    }
  }
  uint64_t stats[4];
  CHECK(nomad_render_stats(ctx, stats));
  std::vector<uint8_t> flags(v.object_count);
  CHECK(nomad_residency_flags(ctx, flags.data()));
  uint64_t resident = 0;
  for (uint32_t o = 0; o < v.object_count; ++o)
    if (flags[o]) resident += bytes[o];
  double sum = 0.0;
  for (float x : radiance) sum += x;
  uint32_t status = 0;
  CHECK(nomad_get_status(ctx, &status));
  if (!a.out.empty()) {
    FILE *f = std::fopen(a.out.c_str(), "wb");
    if (!f) {
      std::fprintf(stderr, "cannot write %s\n", a.out.c_str());
      return 1;
    }
    std::fprintf(f, "PF\n%u %u\n-1.0\n", a.width, a.height);
    for (uint32_t y = a.height; y-- > 0;) std::fwrite(radiance.data() + (size_t)y * a.width * 3, 4, (size_t)a.width * 3, f);
    std::fclose(f);
  }
  const double timed = a.frames > 1 ? (double)(a.frames - 1) : 1.0;
  std::printf(
      "{\"scene\": \"%s\", \"objects\": %u, \"prims\": %u, \"policy\": \"%s\", \"frames\": %u, "
      "\"width\": %u, \"height\": %u, \"spp\": %u, \"depth\": %u, \"render_ms_per_frame\": %.4f, "
      "\"residency_step_ms_per_frame\": %.4f, \"resident_fraction\": %.4f, \"rays\": %llu, "
      "\"shadow_rays\": %llu, \"last_frame\": %u, \"radiance_sum\": %.6f, \"status\": %u, "
      "\"view\": {\"camera_pos\": [%.9g, %.9g, %.9g], \"viewport_u\": [%.9g, %.9g, %.9g], "
      "\"viewport_v\": [%.9g, %.9g, %.9g], \"first_pixel\": [%.9g, %.9g, %.9g]}}\n",
      a.scene.c_str(), v.object_count, v.prim_count, a.policy.c_str(), a.frames, a.width, a.height, a.spp, a.depth,
      render_ms / timed, step_ms / timed, total ? (double)resident / (double)total : 0.0,
      (unsigned long long)stats[0], (unsigned long long)stats[2], a.frames - 1, sum, status, view.camera_pos[0],
      view.camera_pos[1], view.camera_pos[2], view.viewport_u[0], view.viewport_u[1], view.viewport_u[2],
      view.viewport_v[0], view.viewport_v[1], view.viewport_v[2], view.first_pixel[0], view.first_pixel[1],
      view.first_pixel[2]);
  nomad_destroy(ctx);
  nomad_scenebvh_free(bvh);
  if (scene) nomad_scene_owned_free(scene);
  if (loaded) nomad_loaded_scene_free(loaded);
  return status == 0 ? 0 : 1;
}
