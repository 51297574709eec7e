// Per-object residency features, shared by the feature kernel (residency.cu) and the fused
// feature + scorer kernel of the learned policy (mlp.cu).
//
// For object o, one call consumes this frame's closest-hit count, updates the object's hit
// history, decayed ray-hit score, last-hit frame and previous distance, tests the bounding sphere
// against the camera frustum, writes the 24 features and the visibility flag, and returns the
// ray-hit-budget key (RendererResidency.cpp:2833-2840: off-screen objects without hits drop to
// 0, off-screen objects with hits keep lerp(0.5, 0.2, memoryPressure), visible objects with no
// score get 1).
#pragma once
#include <cstdint>

#include "../../../include/nomad_rt.h"

namespace nomad_res {

constexpr int kHist = 8;

struct CamDev {
  float pos[3], fwd[3], right[3], up[3];
  float halfW, halfH, speed;
};

// misc words: [0] toggles, [1] root toggled flag, [2] root resident, [3] total hits this frame,
// [4] total hits previous frame
struct FeatArgs {
  uint32_t n;
  CamDev cam;
  const float4 *bounds;
  const unsigned long long *bytes;
  const uint32_t *tris;
  const float *emit;
  const uint8_t *res;
  uint32_t *hits, *hist;
  float *score;
  uint32_t *lastHit;
  float *prevDist;
  uint8_t *visible;
  float *feat;
  uint32_t *misc;
  uint32_t frame;
  float decay, memPressure;
};

__device__ __forceinline__ float object_features(const FeatArgs &A, uint32_t o, float (&f)[NOMAD_FEATURES]) {
  const CamDev &cam = A.cam;
  const uint32_t frame = A.frame;
  uint32_t h = A.hits[o];
  A.hits[o] = 0;
  if (h) atomicAdd(&A.misc[3], h);
  A.hist[o * kHist + frame % kHist] = h;
  float s = A.score[o] * A.decay + (float)h;
  A.score[o] = s;
  if (h) A.lastHit[o] = frame;
  float4 b = A.bounds[o];
  float dx = b.x - cam.pos[0], dy = b.y - cam.pos[1], dz = b.z - cam.pos[2];
  float dist = sqrtf(dx * dx + dy * dy + dz * dz);
  float z = dx * cam.fwd[0] + dy * cam.fwd[1] + dz * cam.fwd[2];
  float x = dx * cam.right[0] + dy * cam.right[1] + dz * cam.right[2];
  float y = dx * cam.up[0] + dy * cam.up[1] + dz * cam.up[2];
  float r = b.w;
  bool vis = z > -r && fabsf(x) - cam.halfW * z <= r * sqrtf(1.0f + cam.halfW * cam.halfW) &&
             fabsf(y) - cam.halfH * z <= r * sqrtf(1.0f + cam.halfH * cam.halfH);
  A.visible[o] = vis ? 1 : 0;
  float zc = fmaxf(z, 1e-3f);
  f[0] = log1pf(dist);
  f[1] = fminf(r / (fmaxf(dist, 1e-3f) * cam.halfH), 4.0f);
  f[2] = vis ? 1.0f : 0.0f;
#pragma unroll
  for (int k = 0; k < kHist; ++k) f[3 + k] = log1pf((float)A.hist[o * kHist + (frame + kHist - k) % kHist]);
  f[11] = log1pf(s);
  f[12] = log1pf((float)A.tris[o]);
  f[13] = log1pf((float)A.bytes[o] / 1024.0f);
  f[14] = log1pf(A.emit[o]);
  f[15] = cam.speed;
  f[16] = dist > 0.0f ? z / dist : 1.0f;
  f[17] = log1pf(r);
  f[18] = A.res[o] ? 1.0f : 0.0f;
  f[19] = log1pf((float)min(frame - A.lastHit[o], 255u));
  f[20] = (float)h / fmaxf(1.0f, (float)A.misc[4]);
  f[21] = A.prevDist[o] > 0.0f ? A.prevDist[o] - dist : 0.0f;
  f[22] = fminf(fabsf(x) / (zc * cam.halfW), 4.0f);
  f[23] = fminf(fabsf(y) / (zc * cam.halfH), 4.0f);
  A.prevDist[o] = dist;
  float* out = A.feat + (size_t)o * NOMAD_FEATURES;
#pragma unroll
  for (int k = 0; k < NOMAD_FEATURES; ++k) out[k] = f[k];
  float key = s;
  if (!vis) key = (h == 0) ? 0.0f : key * (0.5f + (0.2f - 0.5f) * A.memPressure);
  else if (key <= 0.0f) key = 1.0f;
  return key;
}

}  // namespace nomad_res
