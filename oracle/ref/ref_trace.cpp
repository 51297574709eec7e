// ORACLE glue — test infrastructure only. Runs the reference's own MSL traversal
// (Renderer/Shaders/PathTracing.h: firstHitTLAS / firstHitBVH / intersectAABB, compiled as C++
// through shim/metal_compat.h) over SceneBVH arrays on the host cores. It keeps every quirk of
// the reference: first-found tie rule, per-BLAS best distance, 64-entry stacks that drop
// pushes on overflow, and the leaf-test counter stats[2g+1] incremented before the activeMask
// check.
#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "metal_compat.h"
using namespace metal;
#include "PathTracing.h"
#undef thread
#undef device
#undef constant

extern "C" int ref_trace(const float *bvh, const float *tlas, uint32_t tlasCount, const float *prims,
                         const int32_t *primIndices, const uint8_t *active, const int32_t *blasRoot,
                         const int32_t *primObject, uint32_t primCount, const float *rays,
                         uint64_t n, float *hitsOut, uint32_t *stats, uint32_t threads, int) {
  if (!bvh || !tlas || !prims || !primIndices || !active || !blasRoot || !primObject || !rays || !hitsOut)
    return 1;
  // Instance records as Renderer fills them (blasRootIndex < 0 = not resident).
  uint32_t objCount = 0;
  for (uint32_t p = 0; p < primCount; ++p) objCount = std::max<uint32_t>(objCount, primObject[p] + 1);
  std::vector<InstanceRecord> inst(objCount);
  for (uint32_t o = 0; o < objCount; ++o) inst[o].blasRootIndex = blasRoot[o];
  for (uint32_t p = primCount; p-- > 0;) {
    InstanceRecord &r = inst[primObject[p]];
    r.primitiveBase = p;
    r.primitiveIndexBase = p;
    r.primitiveCount += 1;
  }
  const float4 *B = reinterpret_cast<const float4 *>(bvh);
  const float4 *T = reinterpret_cast<const float4 *>(tlas);
  const float4 *P = reinterpret_cast<const float4 *>(prims);
  atomic_uint *S = reinterpret_cast<atomic_uint *>(stats);
  auto work = [&](uint64_t b, uint64_t e) {
    for (uint64_t i = b; i < e; ++i) {
      const float *q = rays + 8 * i;
      Ray r;
      r.origin = float3(q[0], q[1], q[2]);
      r.direction = float3(q[4], q[5], q[6]);
      r.minDistance = q[3];
      r.maxDistance = q[7];
      intersection h = firstHitTLAS(r, T, tlasCount, B, P, primIndices, active, inst.data(),
                                    nullptr, primCount, primCount, S, nullptr);
      int32_t *o = reinterpret_cast<int32_t *>(hitsOut + 5 * i);
      bool hit = h.primitiveId >= 0;
      o[0] = hit ? primObject[h.primitiveId] : -1;
      o[1] = hit ? h.primitiveId : -1;
      float t = hit ? h.t : INFINITY, u = hit ? h.barycentric.x : 0.0f, v = hit ? h.barycentric.y : 0.0f;
      std::memcpy(o + 2, &t, 4);
      std::memcpy(o + 3, &u, 4);
      std::memcpy(o + 4, &v, 4);
    }
  };
  if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
  if (threads == 1 || n < 1024) {
    work(0, n);
    return 0;
  }
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> pool;
  for (uint32_t t = 0; t < threads; ++t)
    pool.emplace_back([&]() {
      for (;;) {
        uint64_t b = next.fetch_add(256);
        if (b >= n) break;
        work(b, std::min(n, b + 256));
      }
    });
  for (auto &t : pool) t.join();
  return 0;
}
