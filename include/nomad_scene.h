/*
 * nomad_scene.h — host-side scene description and SceneBVH-compatible builder.
 *
 * These entry points replace the host half of the reference's scene pipeline:
 *   - Scene::addObject / addObjectInternal (Nomad Path Tracer/Scene/Scene.cpp:107-168),
 *     including Triangle::computeFrame (Scene/Triangle.h:20-107) and
 *     Rectangle::computeFrame (Scene/Rectangle.h:19-75);
 *   - Scene::buildBVH (Scene/SceneBVH.cpp:16-159) with buildBVHRecursive (:549-623),
 *     evaluateSAHSplit (:704-815) and buildTLASRecursive (:625-702);
 *   - the GPU packers createTransformsBuffer (:165-209), createMaterialsBuffer (:211-222),
 *     createBVHBuffer (:420-428), createTLASBuffer (:467-488) and
 *     createPrimitiveIndexBuffer (:514-520);
 *   - the non-compacted instance-record fill in Renderer::rebuildResidentResources
 *     (Renderer/Renderer.cpp:5305-5326).
 * The arrays they produce use exactly the reference's GPU layouts, so a caller can feed
 * them to nomad_scene_upload (nomad_rt.h) or to any consumer of the reference's buffers.
 *
 * Plus seeded synthetic scene generators (icosphere instances, a procedural city) that
 * stand in for the reference's XML/OBJ scenes.
 *
 * Plus two device stages: the per-object BLAS builds on a CUDA device
 * (nomad_scenebvh_build_gpu) and the compacted residency arrays built on the device
 * (nomad_scenebvh_compact_gpu).
 *
 * All other functions are host-only. All are thread-safe on distinct handles and return
 * nomad_status (0 = OK). No exceptions cross this ABI.
 */
#ifndef NOMAD_SCENE_H
#define NOMAD_SCENE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t nomad_status;
enum {
  NOMAD_OK = 0,
  NOMAD_ERR_INVALID_ARGUMENT = 1,
  NOMAD_ERR_OUT_OF_MEMORY = 2,
  NOMAD_ERR_CUDA = 3,
  NOMAD_ERR_NOT_READY = 4,
  NOMAD_ERR_SCENE_INVALID = 5,
  NOMAD_ERR_DEVICE_STATUS = 6,
  NOMAD_ERR_UNSUPPORTED = 7,
  NOMAD_ERR_LIMIT = 8
};

/* Primitive types, numbered as PrimitiveType (Scene/Primitive.h:13-17). */
enum { NOMAD_PRIM_SPHERE = 0, NOMAD_PRIM_TRIANGLE = 1, NOMAD_PRIM_RECTANGLE = 2 };

/* Floats per primitive in a scene description:
 *   triangle : v0.xyz v1.xyz v2.xyz uv0.xy uv1.xy uv2.xy           (15 used)
 *   rectangle: center.xyz u.xyz v.xyz                               (9 used)
 *   sphere   : center.xyz radius                                    (4 used)            */
#define NOMAD_PRIM_GEOM_FLOATS 15
/* Floats per material = 5 float4, encoded as encodeMaterial (Scene/Material.h:32-44):
 *   {diffuse.rgb, opacity} {specular.rgb, shininess} {emission.rgb, power}
 *   {transmission.rgb, ior} {diffuseTex, specularTex, normalTex, roughness}          */
#define NOMAD_MATERIAL_FLOATS 20
/* float4 per packed primitive and per packed material in the GPU buffers. */
#define NOMAD_PRIM_FLOAT4 7
#define NOMAD_MATERIAL_FLOAT4 5

/* A scene description: primitives grouped into objects. Objects are contiguous,
 * non-overlapping primitive ranges, in order (Scene::addObject appends). */
typedef struct nomad_scene_desc {
  uint32_t prim_count;
  const int32_t *prim_type;      /* [prim_count] NOMAD_PRIM_*                         */
  const float *prim_geom;        /* [prim_count * NOMAD_PRIM_GEOM_FLOATS]             */
  const float *prim_material;    /* [prim_count * NOMAD_MATERIAL_FLOATS]              */
  uint32_t object_count;
  const uint32_t *object_first;  /* [object_count] first primitive of each object     */
  const uint32_t *object_prims;  /* [object_count] primitive count of each object     */
} nomad_scene_desc;

/* The TLAS instance record, laid out as InstanceRecord (Renderer/Shaders/Structs.h:31-37)
 * and BlasInstanceRecord (Renderer/Renderer.h:31-36). blas_root_index < 0 marks an
 * object that is not resident; the traversal skips it. */
typedef struct nomad_instance_record {
  int32_t blas_root_index;
  uint32_t primitive_base;
  uint32_t primitive_count;
  uint32_t primitive_index_base;
} nomad_instance_record;

/* Read-only views of a built SceneBVH. Every pointer stays valid until the handle is freed.
 * Node arrays are float4 pairs: {min.xyz, bits(leftFirst|left)} {max.xyz, bits(count|right)}. */
typedef struct nomad_scenebvh_view {
  uint32_t prim_count;
  uint32_t object_count;
  uint32_t bvh_node_count;       /* BLAS nodes of all objects, concatenated            */
  uint32_t tlas_node_count;
  const float *bvh_nodes;        /* [bvh_node_count * 8]  createBVHBuffer             */
  const float *tlas_nodes;       /* [tlas_node_count * 8] createTLASBuffer            */
  const float *prims;            /* [prim_count * 28]     createTransformsBuffer      */
  const float *materials;        /* [prim_count * 20]     createMaterialsBuffer       */
  const int32_t *prim_indices;   /* [prim_count]          createPrimitiveIndexBuffer  */
  const nomad_instance_record *instances; /* [object_count], all objects resident      */
  const float *object_bounds;    /* [object_count * 6] min.xyz max.xyz                 */
  uint32_t max_depth;            /* deepest TLAS+BLAS root-to-leaf path, in nodes      */
} nomad_scenebvh_view;

typedef struct nomad_scenebvh nomad_scenebvh;

/* Builds the SceneBVH arrays for a scene description (objects in parallel on host
 * threads, like Scene::buildBVH). threads = 0 uses all hardware threads. */
nomad_status nomad_scenebvh_build(const nomad_scene_desc *desc, uint32_t threads,
                                  nomad_scenebvh **out);
/* The same arrays, bit for bit, with the per-object BLAS builds on CUDA device `device`: every
 * node of a tree level (of all objects) is built by one thread block, from the primitive bounds
 * reduction and the 12-bin SAH to the stable sort of the node's primitive range; the TLAS and the
 * packing run on the host as in nomad_scenebvh_build. No counterpart in the reference, which
 * builds BLASes on host threads (Scene::buildBVH). */
nomad_status nomad_scenebvh_build_gpu(const nomad_scene_desc *desc, int32_t device,
                                      nomad_scenebvh **out);
nomad_status nomad_scenebvh_view_get(const nomad_scenebvh *h, nomad_scenebvh_view *out);

/* ---- residency compaction on the device ---- */

/* SceneBVH arrays in device memory, as nomad_scenebvh_view lays them out (every pointer a CUDA
 * device pointer). instances are the full-scene records (every object with primitives has its
 * BLAS root; primitive_base == primitive_index_base == the object's first primitive). */
typedef struct nomad_scenebvh_device {
  uint32_t prim_count;
  uint32_t object_count;
  uint32_t bvh_node_count;
  uint32_t reserved;
  const float *bvh_nodes;                 /* [bvh_node_count * 8]  */
  const float *prims;                     /* [prim_count * 28]     */
  const float *materials;                 /* [prim_count * 20]     */
  const int32_t *prim_indices;            /* [prim_count]          */
  const nomad_instance_record *instances; /* [object_count]        */
} nomad_scenebvh_device;

/* Device output arrays of a compaction, each sized for the full scene (the compact arrays are
 * never longer). counts (device) receives [0] resident primitives, [1] compact BLAS nodes,
 * [2] error bits (0 = OK; 1 index out of range, 2 tree deeper than 128, 4 arrays not laid out
 * as SceneBVH builds them). */
typedef struct nomad_compact_out {
  float *bvh_nodes;                 /* [bvh_node_count * 8] compactBVHNodes             */
  float *prims;                     /* [prim_count * 28]    compactPrimitiveData        */
  float *materials;                 /* [prim_count * 20]    compactMaterialData         */
  int32_t *prim_indices;            /* [prim_count]         compactPrimitiveIndices     */
  uint32_t *remap;                  /* [prim_count]         remapUpload: compact->global */
  int32_t *prim_to_resident;        /* [prim_count]         global->compact, -1 inactive */
  nomad_instance_record *instances; /* [object_count]       compact instance records    */
  uint32_t *counts;                 /* [3]                                              */
} nomad_compact_out;

/* Device scratch bytes nomad_scenebvh_compact_gpu needs for these sizes. */
size_t nomad_compact_workspace_bytes(uint32_t prim_count, uint32_t bvh_node_count, uint32_t object_count);

/* Builds the compacted resident arrays of the reference's compacted residency path
 * (Renderer::rebuildResidentResources, Renderer/Renderer.cpp:5359-5560: active primitives in
 * object and BLAS-leaf order, each object's cached BLAS pruned to its active leaves, one-child
 * nodes collapsed, nodes in post-order with unchanged bounds) from the full arrays and a
 * per-primitive active mask (prim_active[global primitive] != 0), on the device, queued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) without host synchronisation.
 * The TLAS is unchanged. Allocates nothing. Returns NOMAD_ERR_INVALID_ARGUMENT for missing
 * pointers or a workspace smaller than nomad_compact_workspace_bytes; data errors are reported
 * in counts[2]. */
nomad_status nomad_scenebvh_compact_gpu(const nomad_scenebvh_device *in, const uint8_t *prim_active,
                                        void *workspace, size_t workspace_bytes,
                                        const nomad_compact_out *out, void *stream);
void nomad_scenebvh_free(nomad_scenebvh *h);

/* ---- seeded synthetic scenes (no reference counterpart: stand-ins for its XML scenes) ---- */

typedef struct nomad_scene_owned nomad_scene_owned;

/* Small scene: `instances` copies of a 3x-subdivided icosphere (1,280 triangles each),
 * world-space baked with translation U[-extent/2, extent/2]^3, scale U(0.5,3) and a
 * uniform random rotation. One object per instance. */
nomad_status nomad_synth_icospheres(uint64_t seed, uint32_t instances, float extent,
                                    nomad_scene_owned **out);

/* Procedural city: grid x grid_z cells of size_m / grid metres (x spans size_m); each cell is
 * one object holding
 * a noise-displaced box or cylinder with a lognormal triangle count (median
 * `median_tris`, clamped to `max_tris`, rescaled to about `target_tris` in total), its
 * ground tile, and — for `emissive_quads` seeded cells — an emissive rectangle lamp.
 * `emissive_tris` extra small emissive triangles with lognormal power (sigma
 * `emissive_sigma`) are scattered over the roofs (0 for none). */
nomad_status nomad_synth_city(uint64_t seed, uint32_t grid, uint32_t grid_z, float size_m,
                              uint32_t target_tris,
                              uint32_t median_tris, uint32_t max_tris, uint32_t emissive_quads,
                              uint32_t emissive_tris, float emissive_sigma,
                              nomad_scene_owned **out);

nomad_status nomad_scene_owned_desc(const nomad_scene_owned *s, nomad_scene_desc *out);
void nomad_scene_owned_free(nomad_scene_owned *s);

/* ---- scene ingest: the reference's XML scenes with OBJ/MTL meshes ---- */

/* Scene-level settings of a <Scene> root (SceneLoader::LoadSceneFromXML,
 * Scene/SceneLoader.cpp:369-687), with the defaults of Scene::clear (Scene/Scene.cpp:70-101)
 * and ResidencyParameters (Scene/Scene.h). Only the residency parameters of the policies this
 * library implements are carried. */
typedef struct nomad_scene_settings {
  float width, height;              /* screenSize; default 1280 x 720                       */
  uint32_t max_ray_depth;           /* default 32                                           */
  int32_t residency_strategy;       /* ResidencyStrategy numbering (Scene/Scene.h:15-26):
                                       0 DistanceLOD (default), 1 EnergyImportance,
                                       2 RayHitBudget, 3 ScreenSpaceFootprint, 4 Probabilistic,
                                       5 AlwaysResident, 6 EnvironmentHit,
                                       7 PredictiveEnvironment, 8 UnifiedScore, 9 UnifiedNeural */
  int32_t start_compacted;          /* 0/1                                                  */
  int32_t restir_enabled;           /* 0/1                                                  */
  float environment_brightness;     /* default 1                                            */
  uint32_t reserved;
  double texture_cap_mb;            /* textureResidencyMemoryCapMB, default 2048            */
  double geometry_cap_mb;           /* geometryResidencyMemoryCapMB, default 2048           */
  double total_gpu_cap_mb;          /* totalGpuMemoryCapMB, default 4096                    */
  uint64_t max_tile_work;           /* maxTileWork / maxTileWorkPerCommand (at least 1);
                                       default 64 * 64 * 4                                  */
  /* ResidencyParameters read by DistanceLOD, RayHitBudget and ScreenSpaceFootprint */
  float lod_enter_distance, lod_exit_distance;          /* 225, 275                    */
  float lod_enter_view_degrees, lod_exit_view_degrees;  /* 5, 12                       */
  uint32_t state_cooldown_frames;                       /* residencyCooldown, 5        */
  uint32_t ray_hit_cooldown_frames;                     /* rayHitCooldown, 4           */
  uint64_t lod_max_toggles;                             /* lodToggleBudget, 24         */
  float ray_hit_decay, ray_hit_target_fraction;         /* 0.85, 0.54                  */
  uint64_t ray_hit_min_active, ray_hit_max_toggles;     /* 16, 16                      */
  float screen_target_fraction;                         /* screenTargetFraction, 0.68  */
  float screen_min_pixel_coverage;                      /* screenMinPixelCoverage, 32  */
  uint64_t screen_min_active, screen_max_toggles;       /* 16, 14                      */
  float ray_hit_target_memory_mb, screen_target_memory_mb, distance_target_memory_mb;
  float target_memory_mb, target_resident_geometry_mb;  /* all 0 = not given           */
  uint32_t reserved2;
} nomad_scene_settings;

/* <CameraPath><Keyframe …/> (CameraKeyframe, Scene/Scene.h:150-157). */
typedef struct nomad_camera_keyframe {
  uint32_t frame;
  float position[3], look_at[3], up[3];
  float aperture, focus_distance;
} nomad_camera_keyframe;

/* <ObserverCamera …/> (ObserverCamera, Scene/Scene.h:159-166). */
typedef struct nomad_observer_camera {
  float position[3], look_at[3], up[3];
  float vertical_fov, aperture, focus_distance;
} nomad_observer_camera;

typedef struct nomad_loaded_scene nomad_loaded_scene;

typedef struct nomad_loaded_scene_view {
  nomad_scene_desc scene;             /* primitives in load order, objects as added          */
  const int32_t *object_mesh_group;   /* [object_count] meshGroupId; -1 for <Sphere>/<Rectangle> */
  nomad_scene_settings settings;
  uint32_t keyframe_count;
  int32_t has_observer;
  const nomad_camera_keyframe *keyframes;
  nomad_observer_camera observer;
  const char *environment_texture;    /* resolved path, "" when none                         */
  uint32_t mesh_files;                /* distinct OBJ files read                             */
  uint32_t mesh_files_failed;         /* of which failed to parse (loaded as empty meshes)   */
  const char *log;                    /* the loader's warnings, one per line                 */
} nomad_loaded_scene_view;

/* Loads a scene XML and the OBJ/MTL meshes it names into a scene description, like
 * SceneLoader::LoadSceneFromXML (Scene/SceneLoader.cpp:344-858): <Sphere>, <Rectangle> (with
 * Euler XYZ `rotation`), <Mesh> (OBJ world-space baked by position + scale/basis + rotation,
 * material overrides and fallbacks, split into objects by clusterMaxTriangles /
 * clusterMaxExtent), <CameraPath>, <ObserverCamera> and the root's settings. OBJ and MTL
 * parsing follows the vendored tinyobjloader 2.0 (triangulation on: quads split on the shorter
 * diagonal, larger polygons ear-clipped; its own decimal number parser). A mesh file that is
 * missing or fails to parse contributes no triangles, as in the reference. Distinct OBJ files
 * are parsed on `threads` host threads (0 = all hardware threads); the result does not depend
 * on the thread count. Texture images are not decoded: every texture index is -1 (texture
 * residency is not part of this library).
 * Returns NOMAD_ERR_INVALID_ARGUMENT when the XML cannot be read or parsed or has no <Scene>
 * root. */
nomad_status nomad_scene_load_xml(const char *path, uint32_t threads, nomad_loaded_scene **out);
/* Why the calling thread's last failed nomad_scene_load_xml failed ("" after a success); valid
 * until the thread's next call. */
const char *nomad_scene_last_error(void);
nomad_status nomad_loaded_scene_view_get(const nomad_loaded_scene *s, nomad_loaded_scene_view *out);
void nomad_loaded_scene_free(nomad_loaded_scene *s);

#ifdef __cplusplus
}
#endif
#endif
