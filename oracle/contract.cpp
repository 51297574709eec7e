// ORACLE — test infrastructure only. Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference legs may load this library; the product never calls it.
//
// Scalar C++ restatement of the reference's ray traversal over the SceneBVH arrays
// (Nomad Path Tracer/Renderer/Shaders/PathTracing.h), written independently of the CUDA core:
//   intersectAABB      PathTracing.h:646-667
//   firstHitBVH        PathTracing.h:670-959  (triangle :771-848, rectangle :849-913,
//                                              sphere :751-770, activeMask :723)
//   firstHitTLAS       PathTracing.h:961-1066 (instance skip when blasRootIndex < 0 :1005-1006)
// Contract changes from the reference (the CUDA core implements the same contract):
//   (i)   ties in t go to the lowest primitive index instead of the first one found;
//   (ii)  boxes are pruned against best_t * (1 + 2^-10), which makes the closest hit
//         independent of traversal order (a child box lies inside its parent's box, and the
//         slab test is monotone under containment, so only pruning depends on order);
//   (iii) the traversal stack is unbounded (the reference drops pushes past 64, :938-941);
//   (iv)  any-hit is a true any-hit over (1e-4, tmax) with early exit, where the reference's
//         isLightVisible (:503-556) runs a full closest hit and compares ids.
// Three traversal orders are provided and must agree on every ray: the reference order
// (BLAS right child first, TLAS near-first by centre key), near-first by box entry distance
// (the order whose work counters define the algorithmic bytes per ray), and brute force
// (every leaf whose box the ray enters, no pruning).
//
// Arithmetic: float, no fused multiply-add (built with -ffp-contract=off), dot products
// summed as (x + y) + z, normalize(v) = v / sqrt(dot(v, v)).
#include "contract_core.h"

#include <utility>
#include <vector>

using namespace oracle_core;

extern "C" {

// Scene arguments shared by all entry points. prim_object[p] = object of primitive p;
// blas_root[o] < 0 marks a non-resident object; active[p] = 0 skips primitive p.
// mode: 0 reference order, 1 near-first, 2 brute force. threads: 0 = all.
int oracle_trace_closest(const float *bvh, const float *tlas, uint32_t tlas_count,
                         const float *prims, const int32_t *prim_indices, const uint8_t *active,
                         const int32_t *blas_root, const int32_t *prim_object,
                         uint32_t object_count, const float *rays, uint64_t n, float *hits_out,
                         int mode, uint32_t threads) {
  if (!bvh || !tlas || !tlas_count || !prims || !prim_indices || !active || !blas_root ||
      !prim_object || !rays || !hits_out || mode < 0 || mode > 2)
    return 1;
  Job j{{bvh, tlas, tlas_count, prims, prim_indices, active, blas_root, prim_object},
        rays, n, mode, false, object_count, hits_out, nullptr, nullptr};
  run(j, threads);
  return 0;
}

int oracle_trace_any(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                     const int32_t *prim_indices, const uint8_t *active, const int32_t *blas_root,
                     const int32_t *prim_object, uint32_t object_count, const float *rays,
                     uint64_t n, uint8_t *out, int mode, uint32_t threads) {
  if (!bvh || !tlas || !tlas_count || !prims || !prim_indices || !active || !blas_root ||
      !prim_object || !rays || !out || mode < 0 || mode > 2)
    return 1;
  Job j{{bvh, tlas, tlas_count, prims, prim_indices, active, blas_root, prim_object},
        rays, n, mode, true, object_count, nullptr, out, nullptr};
  run(j, threads);
  return 0;
}

// Near-first traversal with work counters (4 words per ray: nodes, tests, instance reads, hit).
int oracle_trace_work(const float *bvh, const float *tlas, uint32_t tlas_count, const float *prims,
                      const int32_t *prim_indices, const uint8_t *active, const int32_t *blas_root,
                      const int32_t *prim_object, uint32_t object_count, const float *rays,
                      uint64_t n, uint32_t *work_out, float *hits_out, uint32_t threads) {
  if (!bvh || !tlas || !tlas_count || !prims || !prim_indices || !active || !blas_root ||
      !prim_object || !rays || !work_out)
    return 1;
  Job j{{bvh, tlas, tlas_count, prims, prim_indices, active, blas_root, prim_object},
        rays, n, 1, false, object_count, hits_out, nullptr, work_out};
  run(j, threads);
  return 0;
}

// Per-object "rays tested": for every ray, every resident object (blas_root >= 0) whose TLAS
// leaf box the segment [1e-4, t_hit[i]] enters (t_hit infinite for a miss), by a test of every
// leaf box (no walk, so no pruning: the device walks the TLAS and relies on a node's box
// containing its children's). counts: object_count words, added to.
int oracle_object_tests(const float *tlas, uint32_t tlas_count, const int32_t *blas_root, uint32_t object_count,
                        const float *rays, const float *t_hit, uint64_t n, uint32_t *counts) {
  if (!tlas || !blas_root || !rays || !t_hit || !counts) return 1;
  std::vector<std::pair<uint32_t, int32_t>> leaves;  // node, object
  for (uint32_t k = 0; k < tlas_count; ++k) {
    const int32_t l = fbits(tlas[8ull * k + 3]);
    if (l < 0) {
      const int32_t obj = -(l + 1);
      if ((uint32_t)obj < object_count && blas_root[obj] >= 0) leaves.push_back({k, obj});
    }
  }
  for (uint64_t i = 0; i < n; ++i) {
    const float *q = rays + 8 * i;
    Ray r{mk(q[0], q[1], q[2]), mk(q[4], q[5], q[6]), t_hit[i]};
    for (const auto &lf : leaves) {
      const float *nd = tlas + 8ull * lf.first;
      if (aabb(r, nd, nd + 4, RAY_EPS, t_hit[i], nullptr)) counts[lf.second]++;
    }
  }
  return 0;
}

}  // extern "C"
