/*
 * nomad_rt.h — C ABI of the B200 traversal / path-tracing core (libnomad_rt.so).
 *
 * The reference binds its hot path as one Metal compute kernel argument table,
 * pathTraceKernel (Nomad Path Tracer/Renderer/Shaders/PathTraceKernel.metal:7-44), filled by
 * Renderer::draw (Renderer/Renderer.cpp:7484-7566), with the C++ residency interface
 * setObjectActive / setPrimitiveActive / updateResidency / flushResidencyChanges above it.
 * Each entry point below names the reference interface it replaces.
 *
 * Conventions
 *   - Every call returns nomad_status (0 = NOMAD_OK; codes in nomad_scene.h). No exceptions
 *     cross the ABI; nomad_last_error() gives the text of the last failure on a context.
 *   - Host pointers unless NOMAD_TRACE_DEVICE_POINTERS is set, in which case the caller passes
 *     CUDA device pointers (e.g. from its own allocator) and the call returns without waiting.
 *   - A context is used from one thread at a time, like the reference's Renderer. Distinct
 *     contexts may run on distinct threads.
 *   - Device-side failures (a traversal stack that would overflow, an exhausted bounded wait)
 *     never fault or trap the GPU: kernels set bits in a status word that nomad_get_status()
 *     returns.
 */
#ifndef NOMAD_RT_H
#define NOMAD_RT_H

#include <stdint.h>
#include <stddef.h>
#include "nomad_scene.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nomad_ctx nomad_ctx;

typedef struct nomad_config {
  int32_t device;          /* CUDA device ordinal                                          */
  uint32_t flags;          /* reserved, 0                                                  */
} nomad_config;

/* One ray: the reference's Ray (Shaders/PathTracing.h:30-35) packed into two float4.
 * Closest-hit accepts t in (RAY_EPS = 1e-4, tmax) and, like firstHitTLAS, does not read tmin;
 * tmax = +inf gives the reference's unbounded closest hit. Any-hit accepts t in (1e-4, tmax). */
typedef struct nomad_ray {
  float ox, oy, oz, tmin;
  float dx, dy, dz, tmax;
} nomad_ray;

/* Closest hit: instance (object) index and primitive index (-1, -1 on a miss), distance t and
 * barycentrics (u, v) of Möller–Trumbore (the reference's intersection.barycentric,
 * Shaders/PathTracing.h:844). Sphere and rectangle hits report u = v = 0. */
typedef struct nomad_hit {
  int32_t inst;
  int32_t prim;
  float t, u, v;
} nomad_hit;

/* Flags of the trace calls. */
enum {
  NOMAD_TRACE_DEVICE_POINTERS = 1u << 0, /* rays/outputs are device pointers                  */
  NOMAD_TRACE_COUNT_HITS = 1u << 1       /* add closest hits to the per-object hit counters   */
};

/* Traversal kernel variants (nomad_autotune picks one per scene; 0 = the tuned or default one).
 * Widths: binary pair nodes (2), 4- and 8-wide nodes collapsed from them. PERSIST: persistent
 * warps take rays 32 at a time from a global cursor. */
enum {
  NOMAD_KERNEL_AUTO = 0,
  NOMAD_KERNEL_BVH2 = 1,
  NOMAD_KERNEL_BVH2_PERSIST = 2,
  NOMAD_KERNEL_BVH4 = 3,
  NOMAD_KERNEL_BVH4_PERSIST = 4,
  NOMAD_KERNEL_BVH8 = 5,
  NOMAD_KERNEL_BVH8_PERSIST = 6,
  NOMAD_KERNEL_COUNT = 7
};

/* ---- context -------------------------------------------------------------------------------- */
nomad_status nomad_create(const nomad_config *cfg, nomad_ctx **out);
nomad_status nomad_destroy(nomad_ctx *ctx);
const char *nomad_last_error(const nomad_ctx *ctx);
/* Waits for all work queued on the context's stream. */
nomad_status nomad_sync(nomad_ctx *ctx);
/* Runs the context's device-pointer work on the caller's CUDA stream (a cudaStream_t passed
 * as void*); NULL restores the context's own stream. */
nomad_status nomad_set_stream(nomad_ctx *ctx, void *cuda_stream);
/* Device status word: bit 0 stack overflow guard, bit 1 bounded wait expired. Cleared by reading. */
nomad_status nomad_get_status(nomad_ctx *ctx, uint32_t *status_word);
/* Self-test of the failure path of the bounded device waits (no counterpart in the reference):
 * one block waits, with a short poll limit, on a shared-memory mbarrier with the helper the
 * traversal's staged-node copy uses. With complete = 0 nothing completes the barrier, the polls
 * run out and bit 1 of the status word is set; otherwise the barrier is completed first and the
 * wait succeeds. The GPU is neither faulted nor held: the kernel returns, the context stays
 * usable. Synchronous on the context's stream. */
nomad_status nomad_selftest_bounded_wait(nomad_ctx *ctx, int32_t complete);

/* ---- scene upload (replaces the GPU uploads of Renderer::rebuildResidentResources,
 *      Renderer.cpp:5983-6292, for the non-compacted resident set) ------------------------ */
/* Arrays use the SceneBVH layouts exactly: bvh_nodes/tlas_nodes are float4 pairs
 * (createBVHBuffer / createTLASBuffer), prims 7 float4 per primitive (createTransformsBuffer),
 * materials 5 float4 per primitive (createMaterialsBuffer), prim_indices int32
 * (createPrimitiveIndexBuffer), instances one record per object. The caller owns the host
 * arrays; the library copies them and builds its traversal layout on the device. All
 * primitives start active; objects with blas_root_index < 0 start non-resident. */
nomad_status nomad_scene_upload(nomad_ctx *ctx, const float *bvh_nodes, uint32_t bvh_node_count,
                                const float *tlas_nodes, uint32_t tlas_node_count,
                                const float *prims, const float *materials,
                                const int32_t *prim_indices, uint32_t prim_count,
                                const nomad_instance_record *instances, uint32_t object_count);

/* ---- residency (Renderer::setPrimitiveActive, Renderer.cpp:7819-7869;
 *      setObjectActive, RendererResidency.cpp:965-1031; flushResidencyChanges,
 *      RendererResidency.cpp:5157-5193) --------------------------------------------------- */
/* Marks one primitive (in)active. *changed = 1 when its state flipped. Takes effect at flush. */
nomad_status nomad_residency_set_primitive_active(nomad_ctx *ctx, uint32_t prim, int32_t active,
                                                  int32_t *changed);
/* Marks every primitive of one object (in)active; *toggled = primitives whose state flipped. */
nomad_status nomad_residency_set_object_active(nomad_ctx *ctx, uint32_t obj, int32_t active,
                                               uint32_t *toggled);
/* Applies pending toggles to the device: an object with no active primitive gets
 * blas_root_index = -1 (skipped by the traversal), inactive primitives are skipped in leaves. */
nomad_status nomad_residency_flush(nomad_ctx *ctx);
/* Copies the current instance records (after the last flush) into out[object_count]. */
nomad_status nomad_residency_get_instances(nomad_ctx *ctx, nomad_instance_record *out);

/* ---- traversal (replaces firstHitTLAS/firstHitBVH, Shaders/PathTracing.h:670-1066, and the
 *      visibility test isLightVisible, :503-556, as standalone ray queries) ---------------- */
/* Closest hit per ray. Ties in t go to the lowest primitive index. */
nomad_status nomad_trace_closest(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n,
                                 nomad_hit *out, uint32_t flags);
/* Any hit per ray in (1e-4, tmax): out[i] = 1 when occluded, else 0. Exits at the first hit. */
nomad_status nomad_trace_any(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n, uint8_t *out,
                             uint32_t flags);
/* Autotuner result: per variant the best of `repeats` closest-hit timings on the sample (ms,
 * negative when the variant is not available for this scene: its stack would be too shallow),
 * the number of sample rays whose hit differs from the binary variant's (must be 0), and the
 * stack entries each width can need on this scene. */
typedef struct nomad_tune_result {
  uint32_t best;                        /* NOMAD_KERNEL_* now used by the context            */
  float ms[NOMAD_KERNEL_COUNT];
  uint32_t mismatches[NOMAD_KERNEL_COUNT];
  uint32_t stack_need[3];               /* binary, 4-wide, 8-wide                            */
} nomad_tune_result;
/* Times every traversal variant on n sample rays (device pointers when
 * NOMAD_TRACE_DEVICE_POINTERS), checks they agree bit for bit, and selects the fastest for the
 * trace calls and the path tracer's queues. */
nomad_status nomad_autotune(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n, uint32_t repeats,
                            uint32_t flags, nomad_tune_result *out);

/* Chooses the traversal variant used by the trace calls (NOMAD_KERNEL_*). */
nomad_status nomad_set_kernel(nomad_ctx *ctx, uint32_t kernel);

/* Full traversal configuration (no counterpart in the reference, which has one kernel). The
 * NOMAD_KERNEL_* variants are the configurations with persistent = 0 or 1. persistent = 2 selects
 * the regrouping kernel, whose persistent warps
 *   - refill idle lanes with new rays from a per-warp pool whenever fewer than `regroup` of the
 *     warp's 32 lanes are still traversing (1: only when the whole warp is idle; 32: as soon as
 *     one lane is idle);
 *   - keep each ray's stack in local memory (short_stack = 0) or its newest `short_stack`
 *     entries in shared memory with older entries spilled to local memory (exact for any depth
 *     the scene needs);
 *   - with postpone_leaves = 1, park the first leaf a lane reaches and keep descending while
 *     other lanes of the warp still look for one, then test the parked leaves together;
 *   - copy the first `staged_nodes` nodes of the layout (the TLAS top levels, numbered
 *     breadth-first) into shared memory with bulk asynchronous copies and read them from there.
 * persistent = 3 selects the hybrid packet kernel: a warp whose 32 rays share an origin and lie in
 * a narrow cone (primary rays) walks the tree as one packet, visiting a node when any lane's ray
 * hits it, with broadcast node and triangle loads; other warps walk per ray.
 * Every configuration returns the same hits bit for bit. */
typedef struct nomad_traversal {
  uint32_t width;           /* 2 (pair nodes), 4 or 8                                          */
  uint32_t persistent;      /* 0: one ray per thread; 1: persistent warps; 2: regrouping warps; */
                            /* 3: hybrid packets (coherent warps walk as one packet)          */
  uint32_t short_stack;     /* persistent = 2: 0 (local memory), 8, 16 or 32                   */
  uint32_t regroup;         /* persistent = 2: refill threshold in busy lanes, 1..32           */
  uint32_t staged_nodes;    /* persistent = 2: top-level nodes staged in shared memory         */
  uint32_t block;           /* threads per block: 0 (default 128), 64, 128, 256                */
  uint32_t postpone_leaves; /* persistent = 2: 1 = park the first leaf and keep descending     */
  uint32_t min_blocks;      /* persistent = 0 or 1: resident blocks per SM the compiler must   */
                            /* fit (0 = no bound; 10, 12 or 16 cap registers for occupancy)    */
} nomad_traversal;
nomad_status nomad_set_traversal(nomad_ctx *ctx, const nomad_traversal *cfg);
nomad_status nomad_get_traversal(nomad_ctx *ctx, nomad_traversal *cfg);
/* Nodes of the TLAS prefix of each layout (widths 2, 4, 8): the most that staging can use. */
nomad_status nomad_tlas_nodes(nomad_ctx *ctx, uint32_t out[3]);

/* One autotuner measurement. */
typedef struct nomad_tune_entry {
  nomad_traversal cfg;
  float ms;               /* best of `repeats` timings; negative when not run                  */
  uint32_t mismatches;    /* sample rays whose hit differs from the binary per-thread kernel's */
} nomad_tune_entry;
/* Sweeps the six NOMAD_KERNEL_* variants, each also with min_blocks 10, 12 and 16, the hybrid
 * packet kernel at widths 2, 4, 8, and, for the regrouping kernel, width {2,4,8} x short
 * stack {0 (local), 8, 16, 32} x regroup threshold {1, 16, 24, 32} x postponed leaves {0, 1} x
 * staged top levels {0, up to 8 KB} x block {128, 256} on n sample rays, checks every
 * configuration against the binary kernel bit for bit, and selects the fastest one that agrees.
 * Fills up to `capacity` entries; *count receives the number of configurations measured. */
nomad_status nomad_autotune_sweep(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n, uint32_t repeats,
                                  uint32_t flags, nomad_tune_entry *entries, uint32_t capacity,
                                  uint32_t *count, nomad_traversal *best);

/* Work counters of a near-first binary traversal over the SceneBVH arrays, per ray:
 * out[4*i+0] nodes whose box was tested (TLAS + BLAS), [1] primitive tests, [2] instance
 * records read, [3] 1 when the ray hit. Defines the algorithmic bytes per ray:
 * 32*nodes + 48*tests + 4*tests + 16*instances + 48*hit. */
nomad_status nomad_trace_work(nomad_ctx *ctx, const nomad_ray *rays, uint64_t n, uint32_t *out,
                              uint32_t flags);

/* ---- hit counters (the reference's primitiveRayStats, Shaders/PathTracing.h:1171-1226, and
 *      the per-object sums of processRayHitCounters, Renderer.cpp:8415-8426) -------------- */
/* Per-object closest-hit counts accumulated by NOMAD_TRACE_COUNT_HITS calls: out[object_count]. */
nomad_status nomad_read_object_hits(nomad_ctx *ctx, uint32_t *out);
nomad_status nomad_reset_object_hits(nomad_ctx *ctx);
/* The same counts into `out[object_count]`, a host array (synchronous) or, with
 * NOMAD_TRACE_DEVICE_POINTERS in flags, a device array (queued on the context's stream). */
nomad_status nomad_read_object_hits_ex(nomad_ctx *ctx, uint32_t *out, uint32_t flags);
/* Replaces the per-object closest-hit counts gathered since the last residency step with
 * `counts[object_count]`, a host array or (NOMAD_TRACE_DEVICE_POINTERS) a device array; queued on
 * the context's stream. No counterpart in the reference, which renders on one GPU: it is the one
 * cross-GPU exchange of a frame split over ranks. Each rank renders its views or tiles with hit
 * counting, the ranks sum the counts (an all-reduce of object_count words), and every rank writes
 * the sum back before its residency step, so all ranks decide the same resident set. */
nomad_status nomad_write_object_hits(nomad_ctx *ctx, const uint32_t *counts, uint32_t flags);

/* ---- path tracing (replaces pathTraceKernel + rayColor, PathTraceKernel.metal:7-162 and
 *      PathTracing.h:1069-1881, as a wavefront loop; the reference's per-pixel seed hash is
 *      replaced by Philox4x32-10 streams) ---------------------------------------------------- */
/* A pinhole view with the reference's uniforms (populateViewportUniforms, Renderer.cpp:1237-1259)
 * plus the frame's sampling parameters. */
typedef struct nomad_view {
  float camera_pos[3];
  float viewport_u[3];
  float viewport_v[3];
  float first_pixel[3];
  uint32_t width, height;
  uint32_t spp;        /* samples (paths) per pixel                                         */
  uint32_t max_depth;  /* closest-hit segments per path (maxRayDepth)                       */
  uint32_t seed_lo, seed_hi; /* Philox key                                                  */
  uint32_t frame;      /* frame index, added to the key's high word                          */
  uint32_t flags;      /* NOMAD_VIEW_*                                                       */
} nomad_view;

enum {
  /* Clamp each sample and each pixel average to [0, 1] like pathTraceKernel (:143) and rayColor
   * (:1879). Without it the output is HDR radiance. */
  NOMAD_VIEW_CLAMP = 1u << 0,
  /* Direct lighting at the first bounce by ReSTIR DI (nomad_set_restir) instead of one-sample NEE. */
  NOMAD_VIEW_RESTIR = 1u << 1,
  /* Primary rays through pixel centres (no sub-pixel jitter). */
  NOMAD_VIEW_CENTER = 1u << 2
};

/* Fills a view from a camera, as populateViewportUniforms does (vertical fov in degrees);
 * spp = 1, max_depth = 1, seeds 0, flags 0. */
nomad_status nomad_view_pinhole(const float position[3], const float look_at[3], const float up[3],
                                float vfov_degrees, uint32_t width, uint32_t height,
                                nomad_view *out);

/* Renders every view in one batched wavefront launch sequence (paths of all views share the
 * ray queues). radiance_out receives RGB floats per pixel, views concatenated
 * (sum of width*height*3 floats); host memory unless NOMAD_TRACE_DEVICE_POINTERS. With
 * NOMAD_TRACE_COUNT_HITS the per-object counters also count the closest hits of every bounce.
 * The frame's launches (raygen, per bounce closest hit, ReSTIR, shading, shadow any-hit,
 * resolve, average) are captured once per frame shape as a CUDA graph and replayed: a shape is
 * the view count, sizes and depths, the output buffer, the traversal configuration, the
 * scene's device arrays and the ReSTIR state. Cameras, seeds and frame numbers are read from
 * the device view table, so they change freely between replays. NOMAD_RENDER_DIRECT launches
 * the same sequence without a graph. */
enum { NOMAD_RENDER_DIRECT = 1u << 2 };
nomad_status nomad_render_frame(nomad_ctx *ctx, const nomad_view *views, uint32_t nviews,
                                float *radiance_out, uint32_t flags);

/* A rectangle of a view's pixels: the reference's TileDispatchRegion (Renderer.cpp:1261-1266),
 * the region its path-tracing kernel renders per dispatch (tile, buffer 16, and
 * pixel = gid + tile.origin, PathTraceKernel.metal:43-58). */
typedef struct nomad_tile {
  uint32_t origin_x, origin_y;
  uint32_t width, height;
} nomad_tile;

/* nomad_render_frame restricted to tiles[i] of views[i] (one tile per view; the tiled dispatch
 * of Renderer.cpp:7319-7581 renders a frame tile by tile). A tile's paths are the view's own
 * paths: the same pixel indices key their random numbers and place their camera rays, so every
 * tile pixel equals that pixel of nomad_render_frame for the same views bit for bit, and with
 * NOMAD_TRACE_COUNT_HITS the per-object counts of tiles that cover a view once add up to the
 * whole frame's. radiance_out receives each tile's pixels row-major, tiles concatenated (sum of
 * width*height*3 floats). A tile must be non-empty and inside its view; a NOMAD_VIEW_RESTIR view
 * must be rendered whole (its reuse reads neighbouring pixels). views[i] is view i of the batch
 * and its index keys its random numbers, as in nomad_render_frame: to reproduce a frame, pass
 * the frame's views in the same order, one tile each, and render further tiles of a view in
 * further calls (a view repeated in one call is another view of the batch, with other samples).
 * Same flags and graph caching as nomad_render_frame. */
nomad_status nomad_render_tiles(nomad_ctx *ctx, const nomad_view *views, const nomad_tile *tiles,
                                uint32_t nviews, float *radiance_out, uint32_t flags);
/* out[0] frame graphs captured, [1] graph launches, [2] graphs cached now (at most 8). */
nomad_status nomad_frame_graph_stats(nomad_ctx *ctx, uint64_t out[3]);

/* ReSTIR DI at the first bounce of views flagged NOMAD_VIEW_RESTIR (replaces the reference's
 * inline reservoir block, PathTracing.h:1363-1742, by separate passes over FP32 reservoirs kept
 * per path (pixel, sample)): `candidates` light samples by RIS (no visibility), temporal reuse
 * of the previous frame's reservoir at the reprojected pixel, `spatial` neighbours drawn within
 * `radius_px` from this frame's temporally resampled reservoirs, each reused reservoir's sample
 * count capped at m_cap * candidates, surface-similarity gates of the reference (position
 * max(1% depth, 0.02), depth max(2% depth, 0.05), normal dot >= 0.9), one visibility ray for the
 * final sample. Temporal reuse needs the same views (sizes, spp) as the previous frame.
 *
 * reference_mode = 1 runs the reference's own ReSTIR instead (PathTracing.h:308-480,
 * :1363-1742): every candidate is traced for visibility before RIS and an occluded or
 * rejected candidate is not counted; the candidate weight is target / solid-angle pdf; reuse
 * reads only the previous frame: its reservoir at the reprojected pixel (temporal, with the
 * reference's Jacobian clamped to 32) and at the 4 pixels +-1 around this one (spatial), each
 * gated by the same surface tests, re-traced for visibility and combined with the reference's
 * MIS weights, uncapped; the result is added without a further visibility ray. `spatial`,
 * `radius_px` and `m_cap` are unused; candidates <= 64. */
typedef struct nomad_restir_config {
  uint32_t candidates;     /* 32                                                           */
  uint32_t temporal;       /* 1 = reuse the previous frame                                 */
  uint32_t spatial;        /* 3 neighbours                                                 */
  float radius_px;         /* 30                                                           */
  float m_cap;             /* 20                                                           */
  uint32_t reference_mode; /* 0 = the configuration above, 1 = the reference's ReSTIR      */
} nomad_restir_config;
nomad_status nomad_set_restir(nomad_ctx *ctx, const nomad_restir_config *cfg);
/* Forgets the previous frame's reservoirs (next frame starts without temporal reuse). */
nomad_status nomad_reset_restir(nomad_ctx *ctx);

/* Ray statistics accumulated by nomad_render_frame since the last reset:
 * out[0] closest-hit rays traced, [1] environment escapes (the reference's stats[2N]),
 * [2] shadow rays traced, [3] closest hits. */
nomad_status nomad_render_stats(nomad_ctx *ctx, uint64_t out[4]);
nomad_status nomad_reset_render_stats(nomad_ctx *ctx);

/* ---- residency policies on the device (updateResidency, RendererResidency.cpp:165-287, with
 *      updateAlwaysResident :656-728, updateRayHitBudget :2755-2964 and the learned scorer that
 *      replaces updateUnifiedResidency/UnifiedNeural :2331-2753) ---------------------------- */
enum {
  NOMAD_POLICY_ALWAYS = 0,        /* every object resident (the image judge)                  */
  NOMAD_POLICY_RAYHIT_BUDGET = 1, /* decayed per-object closest-hit score (the fallback)       */
  NOMAD_POLICY_LEARNED = 2,       /* BF16 MLP score over NOMAD_FEATURES per-object features    */
  NOMAD_POLICY_RAYHIT_PRIM = 3,   /* the reference's per-primitive ray-hit budget (see below)    */
  NOMAD_POLICY_DISTANCE_LOD = 4,  /* the reference's DistanceLOD heuristic (see below)           */
  NOMAD_POLICY_SCREEN_SPACE = 5,  /* the reference's ScreenSpaceFootprint heuristic (see below)  */
  NOMAD_POLICY_PROBABILISTIC = 6, /* the reference's Probabilistic heuristic (see below)         */
  NOMAD_POLICY_ENVIRONMENT_HIT = 7, /* the reference's EnvironmentHit heuristic (see below)      */
  NOMAD_POLICY_PREDICTIVE = 8,    /* the reference's PredictiveEnvironment heuristic (see below) */
  NOMAD_POLICY_ENERGY = 9         /* the reference's EnergyImportance heuristic (see below)      */
};
#define NOMAD_FEATURES 24

typedef struct nomad_residency_params {
  uint32_t policy;
  uint32_t max_toggles;     /* residency changes applied per step; 0 = unlimited             */
  uint64_t budget_bytes;    /* geometry bytes allowed resident; 0 = no limit                 */
  float hit_decay;          /* score = score * hit_decay + hits (rayHitDecay, 0.85)          */
  float camera_motion;      /* [0,1]: widens the visibility reserve                          */
  float memory_pressure;    /* [0,1]: off-screen objects with hits keep lerp(0.5,0.2,p)      */
  float reserve_base;       /* visibility reserve = ceil(N * (base + motion * reserve_motion)) */
  float reserve_motion;
  uint32_t min_active;      /* objects always kept (highest scores first); primitives for
                               NOMAD_POLICY_RAYHIT_PRIM (rayHitMinActivePrimitives, 16)        */
  /* NOMAD_POLICY_RAYHIT_PRIM only (rayHitTargetFraction 0.54, rayHitRebuildCooldownFrames 4,
   * stateCooldownFrames 5; max_toggles is rayHitMaxTogglesPerFrame, 16, 0 = unlimited): */
  float target_fraction;    /* primitives kept = ceil(N * clamp(f + 0.1 motion - 0.24 pressure, 0.34, 0.92)) */
  uint32_t rebuild_cooldown;/* steps skipped after a step that changed residency              */
  uint32_t state_cooldown;  /* steps a toggled primitive stays as it is                       */
  /* NOMAD_POLICY_DISTANCE_LOD only (lodEnterDistance 225, lodExitDistance 275,
   * lodEnterViewDegrees 5, lodExitViewDegrees 12; max_toggles is lodMaxTogglesPerFrame, 24;
   * state_cooldown is the object cooldown): */
  float lod_enter_distance, lod_exit_distance;
  float lod_enter_view_degrees, lod_exit_view_degrees;
  /* NOMAD_POLICY_SCREEN_SPACE only (screenFootprintMinPixelCoverage 32; target_fraction is
   * screenFootprintTargetFraction 0.68, min_active screenFootprintMinActivePrimitives 16,
   * max_toggles screenFootprintMaxTogglesPerFrame 14, in primitives): */
  float min_pixel_coverage;
  /* The per-object Beta hit-probability posterior that every device step updates
   * (processRayHitCounters, Renderer.cpp:8004-8522): alpha, beta decay by probability_decay and
   * gain the step's closest hits and misses (rays tested - hits); a step without tested rays cools
   * the probability (optionally with a grace of probability_idle_frames steps at
   * probability_idle_decay for visible or resident objects); the mass alpha + beta stays in
   * [1e-3, probability_window] (0 = no upper clamp). "Rays tested" of an object: closest-hit ray
   * segments [1e-4, t of the hit] that enter its TLAS leaf box (the reference counts leaf
   * primitive tests, which depend on the traversal order), counted by render and trace calls with
   * NOMAD_TRACE_COUNT_HITS once a step has asked for them (NOMAD_POLICY_PROBABILISTIC, or a
   * ray-hit prior). Defaults: probabilityDecay 0.9, probabilityEvidenceWindow 64,
   * probabilityIdleCooldownFrames 0, probabilityIdleDecay 0.9, probabilityThreshold 0.5. */
  float probability_decay;
  float probability_window;
  uint32_t probability_idle_frames;
  float probability_idle_decay;
  float probability_threshold;
  /* NOMAD_POLICY_RAYHIT_BUDGET: the reference's ray-hit prior (enableRayHitPrior,
   * RendererResidency.cpp:2842-2861): every key times clamp(1 + (p - 0.5) * scale, 0.25, 1) with
   * p the object's hit probability. The reference's default is rayHitPriorScale 0.5; 0 = off. */
  float rayhit_prior_scale;
  /* NOMAD_POLICY_PROBABILISTIC only (updateProbabilisticResidency, RendererResidency.cpp:3389-4090,
   * one object at a time; target_fraction is probabilityTargetFraction 0.60, min_active
   * probabilityMinActivePrimitives 16 and max_toggles probabilityMaxTogglesPerFrame 20, both in
   * primitives; state_cooldown the object cooldown, stateCooldownFrames 5): */
  float uncertainty_boost;           /* probabilityUncertaintyBoost 0.25                       */
  float desired_hysteresis;          /* probabilityDesiredHysteresis 0.02                      */
  float visible_floor;               /* probabilityVisibleFloor 0                              */
  uint32_t recent_promotion_frames;  /* probabilityRecentPromotionFrames 4                     */
  uint32_t demotion_dwell_frames;    /* probabilityVisibleDemotionDwellFrames 0                */
  /* NOMAD_POLICY_ENVIRONMENT_HIT and NOMAD_POLICY_PREDICTIVE (updateEnvironmentHitResidency,
   * RendererResidency.cpp:4759-5155; updatePredictiveResidency :4397-4757; target_fraction is
   * environmentTargetActiveFraction 0.25, min_active environmentMinActivePrimitives 16 and
   * max_toggles environmentMaxTogglesPerFrame 20, in primitives): */
  float env_escape_threshold;        /* environmentEscapeThreshold 0.4                         */
  float env_high_escape;             /* envHighEscapeThreshold 0.6 (EnvironmentHit only)       */
  float env_low_escape;              /* envLowEscapeThreshold 0.3 (EnvironmentHit only)        */
  /* NOMAD_POLICY_ENERGY (updateEnergyImportance, RendererResidency.cpp:1344-1860, scenes without
   * mesh groups; target_fraction is energyTargetFraction 0.88, min_active
   * energyMinActivePrimitives 16, max_toggles energyMaxTogglesPerFrame 32, in primitives;
   * state_cooldown both the object cooldown and the minimum duration between an object's
   * residency changes, stateCooldownFrames 5): */
  float energy_visibility_boost;     /* energyVisibilityBoost 1.75                             */
  float energy_smoothing;            /* energyImportanceSmoothing 0.85                         */
  uint32_t energy_use_average;       /* energyUseAverageImportance 1                           */
  /* NOMAD_POLICY_RAYHIT_BUDGET and NOMAD_POLICY_LEARNED: hysteresis of the selection. A resident
   * object's key k becomes k + resident_key_bonus * |k| before the sort, so it leaves the resident
   * set only for an object that scores that much higher. Each re-entry of an evicted object costs
   * an onload when geometry is paged, so this trades a little image error for fewer copies.
   * No counterpart in the reference, whose ray-hit step has rebuild and state cooldowns instead;
   * 0 = off. */
  float resident_key_bonus;
} nomad_residency_params;

/* One residency step, all on the device: consumes the per-object closest-hit counts gathered
 * since the previous step (render or trace calls with NOMAD_TRACE_COUNT_HITS), updates the
 * per-object history and the NOMAD_FEATURES features for `camera`, scores every object with the
 * policy, selects the resident set greedily by score under budget_bytes (visible objects first
 * up to the visibility reserve, ties to the lower object index), and patches the TLAS so
 * non-resident objects are skipped (blas_root_index = -1). The light CDF follows the resident
 * set. *toggled receives the number of objects whose residency changed; the call then waits for
 * the step. With toggled = NULL the step is queued on the context's stream without any host
 * synchronisation (the host-side residency state is refreshed when a residency call next reads
 * it). Object geometry bytes = 32 per BLAS node + 196 per primitive (packed primitive, material
 * and index). */
nomad_status nomad_residency_step(nomad_ctx *ctx, const nomad_residency_params *params,
                                  const nomad_view *camera, uint32_t *toggled);
/* The per-object hit-probability posterior after the last step (the reference's _objectHitAlpha,
 * _objectHitBeta, _objectHitProbability, _objectHitVariance, _objectPosteriorMass,
 * _objectExplorationScore, _objectIdleFrames, _objectHitLastFrame, _objectRaysTestedLastFrame):
 * 9 words per object, 6 float32 then 3 uint32. */
nomad_status nomad_residency_posterior(nomad_ctx *ctx, float *out);
/* Switches the per-object "rays tested" counting of render and trace calls with
 * NOMAD_TRACE_COUNT_HITS on or off (steps that need it switch it on themselves). tests (may be
 * NULL) receives the counts gathered since the last step or read, which are then cleared. */
nomad_status nomad_residency_count_tests(nomad_ctx *ctx, int32_t on, uint32_t *tests);
/* NOMAD_POLICY_RAYHIT_PRIM restates updateRayHitBudget per primitive, as the reference runs it
 * (RendererResidency.cpp:2755-2964, with the per-frame cooldown decrement of :205-207): per-primitive
 * closest hits (counted by nomad_render_frame with NOMAD_TRACE_COUNT_HITS once the policy has run
 * a step) decay into a score (score * hit_decay + hits), off-screen primitives (bounding sphere
 * outside the camera frustum) keep nothing without hits and lerp(0.5, 0.2, pressure) of their
 * score with hits, visible ones at least 1; the top target by (score, lower index) are wanted,
 * plus the best visible up to ceil(N * (0.02 + 0.06 motion)) and the min_active best; toggles
 * go in primitive order, skip primitives in their cooldown and stop at
 * max(1, round(max_toggles * (1 + 0.45 motion + 0.6 pressure))). It runs on the host over the
 * device's counters and applies its toggles with nomad_residency_set_primitive_active and
 * nomad_residency_flush (toggled != NULL is required). For the host-side policies *toggled
 * counts primitives (NOMAD_POLICY_RAYHIT_PRIM, NOMAD_POLICY_SCREEN_SPACE) or objects
 * (NOMAD_POLICY_DISTANCE_LOD) toggled. */
/* NOMAD_POLICY_DISTANCE_LOD restates updateLODByDistance (RendererResidency.cpp:759-964): each
 * object's bounding sphere (centre and half diagonal of its BLAS root box, Renderer.cpp:3272-3278)
 * gives a distance (to the sphere, 0 inside, none behind the camera) and an angular frustum test
 * with an entry and a wider exit margin; objects are visited nearest first and an inactive one is
 * activated closer than lod_enter_distance inside the entry frustum, an active one kept up to
 * lod_exit_distance inside the exit frustum, objects in their cooldown skipped, at most
 * max(1, round(max_toggles * (1 + 0.4 motion + 0.6 pressure))) toggles. Host-side like the
 * reference, applied with nomad_residency_set_object_active + nomad_residency_flush (toggled
 * != NULL is required). */
/* NOMAD_POLICY_SCREEN_SPACE restates updateScreenSpaceFootprint (RendererResidency.cpp:4092-4396)
 * with every object its own mesh group: each object's projected bounding-sphere area in pixels
 * (0 outside the view, scaled by the cosine to the view axis, at most the screen), objects taken
 * by coverage (ties to the lower index) until min_active primitives and
 * clamp(target_fraction + 0.08 motion - 0.10 pressure, 0.5, 0.94) of the screen are covered,
 * skipping objects under min_pixel_coverage once min_active is met; toggles in coverage order
 * while fewer than max(1, round(max_toggles * (1 + 0.4 motion + 0.5 pressure))) primitives have
 * been toggled, objects or primitives in their cooldown blocking. Host-side; the last step's
 * coverage is returned by nomad_residency_object_state as `distance`. */
/* The DistanceLOD state after its last step, per object (any may be NULL): distance (float,
 * FLT_MAX behind the camera), flags (uint8: 1 entry frustum, 2 exit frustum, 4 behind) and
 * cooldowns (uint32). */
nomad_status nomad_residency_object_state(nomad_ctx *ctx, float *distance, uint8_t *flags, uint32_t *cooldowns);
/* Per-primitive closest hits counted since the last step (prim_count uint32), and the
 * per-primitive policy's state after its last step: decayed scores (float), cooldowns (uint32),
 * the frustum test of that step (uint8, isInView, Renderer.cpp:1765-1817), and every primitive's
 * activity (uint8); any may be NULL. */
nomad_status nomad_residency_prim_state(nomad_ctx *ctx, uint32_t *hits, float *scores, uint32_t *cooldowns,
                                        uint8_t *visible, uint8_t *active);
/* Per-object geometry bytes (object_count uint64). */
nomad_status nomad_object_bytes(nomad_ctx *ctx, uint64_t *out);
/* Features and policy scores of the last step: features[object_count * NOMAD_FEATURES],
 * scores[object_count] (either may be NULL). */
nomad_status nomad_residency_last(nomad_ctx *ctx, float *features, float *scores);
/* Current residency of each object (object_count bytes, 1 = resident). */
nomad_status nomad_residency_flags(nomad_ctx *ctx, uint8_t *out);
/* NOMAD_POLICY_LEARNED falls back to NOMAD_POLICY_RAYHIT_BUDGET (the same step with the same
 * parameters) whenever the context holds no usable model: none initialised, set, trained or
 * loaded yet, or the last nomad_mlp_set / nomad_mlp_load was rejected. The north star's fallback
 * for a model that fails to load, in place of the reference's heuristic unified score
 * (RendererUnifiedNeural.cpp:402-417). *out receives the number of steps that fell back since
 * the scene was uploaded. */
nomad_status nomad_residency_fallback_steps(nomad_ctx *ctx, uint64_t *out);

/* ---- geometry paging (the Cold -> Streaming -> Resident lifecycle of per-object GPU
 *      resources, Renderer.h:63-106, ensureResident Renderer.cpp:613-650, the per-frame onload
 *      loop with kMaxColdObjectOnloadsPerFrame Renderer.cpp:5828-5905) -------------------------
 * Once enabled, every object's BLAS nodes (of the one traversal layout named by `width`) and
 * triangle records live in pinned host memory and are streamed on demand into a fixed device
 * pool of pool_bytes: a Cold object that the residency state wants resident is copied by the
 * copy engine (asynchronously, at most max_onloads_per_frame objects started per update),
 * relocated on the device to its pool offsets, and published into the TLAS when its copy has
 * completed (Streaming -> Resident); an object no longer wanted is unlinked at once and its
 * copy kept as a cache (Cached) until an onload needs the space, which is reused after the work
 * queued before the unlink has finished. An onload that does not fit even after the cache is
 * released is denied (the reference's geometry hard cap). Until an object is
 * Resident it is skipped by traversal even if its residency flag is set. The TLAS and the
 * shading arrays (packed primitives, materials) stay resident. Traversal configurations of
 * other widths, nomad_trace_work and the allocation-free call need the pair layout and are
 * refused while paging a wide layout. Paging lasts until the next nomad_scene_upload; every
 * trace, render and residency call must use the context's stream. */
typedef struct nomad_paging_config {
  uint64_t pool_bytes;            /* device bytes for BLAS nodes + triangle records           */
  uint32_t max_onloads_per_frame; /* Cold objects started per update; 0 = 32 (the reference's) */
  uint32_t width;                 /* paged node layout: 2 (pair), 4 or 8                      */
} nomad_paging_config;

/* CACHED: no longer wanted, unlinked, but its pool copy is kept until the space is needed (least
 * recently unwanted first), so an object the residency state wants back is relinked without a
 * copy and without counting against the onload cap. */
enum { NOMAD_PAGE_COLD = 0, NOMAD_PAGE_STREAMING = 1, NOMAD_PAGE_RESIDENT = 2, NOMAD_PAGE_CACHED = 3 };

typedef struct nomad_paging_stats {
  uint64_t pool_bytes;            /* node + record pool capacity                              */
  uint64_t used_bytes;            /* pool bytes held by Streaming and Resident objects        */
  uint64_t full_bytes;            /* bytes the whole scene's BLAS nodes + records take        */
  uint64_t bytes_streamed;        /* host -> device bytes of all onloads                      */
  uint32_t cold, streaming, resident;
  uint32_t onloads, evictions, denied, deferred; /* totals since enable                       */
  uint32_t cached;                /* objects in NOMAD_PAGE_CACHED                              */
  uint32_t relinks;               /* cached objects wanted again and relinked (total)          */
} nomad_paging_stats;

nomad_status nomad_paging_enable(nomad_ctx *ctx, const nomad_paging_config *cfg);
/* Applies the current residency state (after nomad_residency_flush or nomad_residency_step):
 * publishes completed onloads, unlinks unwanted objects, starts new onloads. Does not wait for
 * copies; call once per frame. */
nomad_status nomad_paging_update(nomad_ctx *ctx);
/* Waits for the copies in flight and publishes them (does not start new onloads). */
nomad_status nomad_paging_wait(nomad_ctx *ctx);
/* on != 0: every nomad_paging_update first waits for the copies the previous updates started and
 * for the frames that unlinked released pool space, then publishes and reuses all of them, so
 * which objects a frame traces depends only on the sequence of calls, not on how fast the copies
 * ran: runs repeat exactly. It costs a host wait when a copy is still in flight (a frame loop that
 * waits for its frame anyway loses nothing). on = 0 (the default): an update publishes what has
 * completed, as the reference's streaming does, and runs can differ by copy timing. No
 * counterpart in the reference. */
nomad_status nomad_paging_set_sync(nomad_ctx *ctx, int32_t on);
nomad_status nomad_paging_stats_get(nomad_ctx *ctx, nomad_paging_stats *out);
/* Per-object NOMAD_PAGE_* state (object_count bytes). */
nomad_status nomad_paging_states(nomad_ctx *ctx, uint8_t *out);

/* ---- learned scorer: 24 -> 128 -> 128 -> 1 MLP, ReLU, BF16 weights, FP32 accumulation on the
 *      tensor cores, trained on device (no reference counterpart for the kernels; the reference
 *      trains a tiny FP32 MLP offline in PyTorch, Benchmarks/train_unified_neural_mlp.py) ---- */
#define NOMAD_MLP_PARAMS (128 * 32 + 128 + 128 * 128 + 128 + 128 + 1 + 2 * NOMAD_FEATURES)
/* Initialises the weights (He-uniform) from a seed. */
nomad_status nomad_mlp_init(nomad_ctx *ctx, uint64_t seed);
/* Trains on n samples (features n*NOMAD_FEATURES, targets n, host arrays): standardises the
 * features, then `steps` AdamW steps of mean-squared error on mini-batches of `batch` samples
 * drawn with a seeded permutation (beta 0.9 / 0.999, eps 1e-8, decoupled weight decay on the
 * weights, not the biases). Each call starts a fresh optimiser state (zero moments) from the
 * current weights. loss_out[steps] (may be NULL) receives each step's loss. */
nomad_status nomad_mlp_train(nomad_ctx *ctx, const float *features, const float *targets, uint64_t n,
                             uint32_t steps, uint32_t batch, float lr, float weight_decay, uint64_t seed,
                             float *loss_out);
/* The mean-squared-error gradient of the current model over n samples taken in order (host
 * arrays; n a multiple of 64, at most 65,536), with the model's stored feature statistics, by
 * the same forward and backward kernels as one training step: grad[NOMAD_MLP_PARAMS] in the
 * blob's layout (0 for W1's padded columns and the statistics), *loss (may be NULL) the mean
 * squared error. For gradient checks of the training kernels. */
nomad_status nomad_mlp_gradient(nomad_ctx *ctx, const float *features, const float *targets, uint64_t n,
                                float *grad, float *loss);
/* Inference on n samples (host arrays unless NOMAD_TRACE_DEVICE_POINTERS). */
nomad_status nomad_mlp_infer(nomad_ctx *ctx, const float *features, uint64_t n, float *out, uint32_t flags);
/* Model blob (NOMAD_MLP_PARAMS floats): W1[128][32] (inputs padded to 32), b1, W2[128][128],
 * b2, w3[128], b3, feature mean[24], feature inverse std[24]. Checkpoint and restore. */
nomad_status nomad_mlp_get(nomad_ctx *ctx, float *out);
/* A blob with a non-finite value is rejected (NOMAD_ERR_INVALID_ARGUMENT) and leaves the context
 * without a usable model, so learned steps fall back to the ray-hit budget until a valid one is
 * set. */
nomad_status nomad_mlp_set(nomad_ctx *ctx, const float *in);
/* The model as a versioned file (the checkpoint the reference keeps as a JSON model file,
 * export_unified_neural_model.py): "NMLP", format version 1, NOMAD_MLP_PARAMS and NOMAD_FEATURES
 * (uint32 little-endian each), the blob (float32 little-endian), then a 64-bit FNV-1a checksum
 * of everything before it. nomad_mlp_load checks every field, the size, the checksum and that
 * every value is finite; on any failure it returns NOMAD_ERR_INVALID_ARGUMENT with the reason
 * in nomad_last_error and leaves the context without a usable model (learned steps then fall
 * back to the ray-hit budget). */
nomad_status nomad_mlp_save(nomad_ctx *ctx, const char *path);
nomad_status nomad_mlp_load(nomad_ctx *ctx, const char *path);

/* ---- allocation-free closest hit (no counterpart in the reference) ----------------------
 * For callers that cannot allocate GPU memory while tracing: a frame loop whose memory budget
 * is fully committed to resident geometry, or one that cannot take the implicit device
 * synchronisation cudaMalloc/cudaFree may cause mid-frame. Same result as nomad_trace_closest
 * with NOMAD_TRACE_COUNT_HITS on device pointers, but its scratch (work cursor + per-object hit
 * accumulators) is a fixed static device array, so the call allocates nothing:
 *   - d_rays[n] in, d_hits[n] and d_object_hits[object_count] (hits of this call only) out,
 *     all device pointers; asynchronous on the context's stream;
 *   - scenes with more than 16,384 objects are rejected (NOMAD_ERR_LIMIT);
 *   - the first call on a device looks up the static array's address; make it before any
 *     stream capture. The array stays allocated on every GPU that loads the library;
 *   - all calls share the array: calls that overlap on the GPU race. Serialise them. */
nomad_status nomad_trace_closest_noalloc(nomad_ctx *ctx, const nomad_ray *d_rays, uint64_t n,
                                         nomad_hit *d_hits, uint32_t *d_object_hits);

#ifdef __cplusplus
}
#endif
#endif
