"""ctypes bindings for libnomad_rt.so (include/nomad_rt.h, include/nomad_scene.h).

The library is built in-tree (``make -C nomad_b200/csrc``) and loaded from
``nomad_b200/lib/libnomad_rt.so``. Importing this module never falls back to anything else:
when the library is missing, :func:`load` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libnomad_rt.so")

NOMAD_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "OUT_OF_MEMORY", 3: "CUDA", 4: "NOT_READY",
    5: "SCENE_INVALID", 6: "DEVICE_STATUS", 7: "UNSUPPORTED", 8: "LIMIT",
}
PRIM_SPHERE, PRIM_TRIANGLE, PRIM_RECTANGLE = 0, 1, 2
TRACE_DEVICE_POINTERS = 1 << 0
TRACE_COUNT_HITS = 1 << 1
KERNEL_AUTO, KERNEL_BVH2, KERNEL_BVH2_PERSIST = 0, 1, 2

# numpy views of the ABI structs
RAY_DTYPE = np.dtype([("ox", "<f4"), ("oy", "<f4"), ("oz", "<f4"), ("tmin", "<f4"),
                      ("dx", "<f4"), ("dy", "<f4"), ("dz", "<f4"), ("tmax", "<f4")])
HIT_DTYPE = np.dtype([("inst", "<i4"), ("prim", "<i4"), ("t", "<f4"), ("u", "<f4"), ("v", "<f4")])
INSTANCE_DTYPE = np.dtype([("blas_root_index", "<i4"), ("primitive_base", "<u4"),
                           ("primitive_count", "<u4"), ("primitive_index_base", "<u4")])


class NomadError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"nomad status {status} ({STATUS_NAMES.get(status, '?')}): {message}")


class SceneDesc(C.Structure):
    _fields_ = [("prim_count", C.c_uint32), ("prim_type", C.POINTER(C.c_int32)),
                ("prim_geom", C.POINTER(C.c_float)), ("prim_material", C.POINTER(C.c_float)),
                ("object_count", C.c_uint32), ("object_first", C.POINTER(C.c_uint32)),
                ("object_prims", C.POINTER(C.c_uint32))]


class SceneSettings(C.Structure):
    """nomad_scene_settings: a <Scene> root's settings (defaults of the reference's Scene)."""
    _fields_ = [("width", C.c_float), ("height", C.c_float), ("max_ray_depth", C.c_uint32),
                ("residency_strategy", C.c_int32), ("start_compacted", C.c_int32), ("restir_enabled", C.c_int32),
                ("environment_brightness", C.c_float), ("reserved", C.c_uint32),
                ("texture_cap_mb", C.c_double), ("geometry_cap_mb", C.c_double), ("total_gpu_cap_mb", C.c_double),
                ("max_tile_work", C.c_uint64),
                ("lod_enter_distance", C.c_float), ("lod_exit_distance", C.c_float),
                ("lod_enter_view_degrees", C.c_float), ("lod_exit_view_degrees", C.c_float),
                ("state_cooldown_frames", C.c_uint32), ("ray_hit_cooldown_frames", C.c_uint32),
                ("lod_max_toggles", C.c_uint64), ("ray_hit_decay", C.c_float), ("ray_hit_target_fraction", C.c_float),
                ("ray_hit_min_active", C.c_uint64), ("ray_hit_max_toggles", C.c_uint64),
                ("screen_target_fraction", C.c_float), ("screen_min_pixel_coverage", C.c_float),
                ("screen_min_active", C.c_uint64), ("screen_max_toggles", C.c_uint64),
                ("ray_hit_target_memory_mb", C.c_float), ("screen_target_memory_mb", C.c_float),
                ("distance_target_memory_mb", C.c_float), ("target_memory_mb", C.c_float),
                ("target_resident_geometry_mb", C.c_float), ("reserved2", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.startswith("reserved")}


class CameraKeyframe(C.Structure):
    _fields_ = [("frame", C.c_uint32), ("position", C.c_float * 3), ("look_at", C.c_float * 3),
                ("up", C.c_float * 3), ("aperture", C.c_float), ("focus_distance", C.c_float)]


class ObserverCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3),
                ("vertical_fov", C.c_float), ("aperture", C.c_float), ("focus_distance", C.c_float)]


class LoadedSceneView(C.Structure):
    _fields_ = [("scene", SceneDesc), ("object_mesh_group", C.POINTER(C.c_int32)), ("settings", SceneSettings),
                ("keyframe_count", C.c_uint32), ("has_observer", C.c_int32),
                ("keyframes", C.POINTER(CameraKeyframe)), ("observer", ObserverCamera),
                ("environment_texture", C.c_char_p), ("mesh_files", C.c_uint32), ("mesh_files_failed", C.c_uint32),
                ("log", C.c_char_p)]


class SceneBVHView(C.Structure):
    _fields_ = [("prim_count", C.c_uint32), ("object_count", C.c_uint32),
                ("bvh_node_count", C.c_uint32), ("tlas_node_count", C.c_uint32),
                ("bvh_nodes", C.POINTER(C.c_float)), ("tlas_nodes", C.POINTER(C.c_float)),
                ("prims", C.POINTER(C.c_float)), ("materials", C.POINTER(C.c_float)),
                ("prim_indices", C.POINTER(C.c_int32)), ("instances", C.c_void_p),
                ("object_bounds", C.POINTER(C.c_float)), ("max_depth", C.c_uint32)]


class ScenebvhDevice(C.Structure):
    """nomad_scenebvh_device: SceneBVH arrays in device memory."""
    _fields_ = [("prim_count", C.c_uint32), ("object_count", C.c_uint32), ("bvh_node_count", C.c_uint32),
                ("reserved", C.c_uint32), ("bvh_nodes", C.c_void_p), ("prims", C.c_void_p),
                ("materials", C.c_void_p), ("prim_indices", C.c_void_p), ("instances", C.c_void_p)]


class CompactOut(C.Structure):
    """nomad_compact_out: device output arrays of a residency compaction."""
    _fields_ = [("bvh_nodes", C.c_void_p), ("prims", C.c_void_p), ("materials", C.c_void_p),
                ("prim_indices", C.c_void_p), ("remap", C.c_void_p), ("prim_to_resident", C.c_void_p),
                ("instances", C.c_void_p), ("counts", C.c_void_p)]


class PagingConfig(C.Structure):
    _fields_ = [("pool_bytes", C.c_uint64), ("max_onloads_per_frame", C.c_uint32), ("width", C.c_uint32)]


class PagingStats(C.Structure):
    _fields_ = [("pool_bytes", C.c_uint64), ("used_bytes", C.c_uint64), ("full_bytes", C.c_uint64),
                ("bytes_streamed", C.c_uint64), ("cold", C.c_uint32), ("streaming", C.c_uint32),
                ("resident", C.c_uint32), ("onloads", C.c_uint32), ("evictions", C.c_uint32),
                ("denied", C.c_uint32), ("deferred", C.c_uint32), ("cached", C.c_uint32),
                ("relinks", C.c_uint32)]


PAGE_COLD, PAGE_STREAMING, PAGE_RESIDENT, PAGE_CACHED = 0, 1, 2, 3


class Config(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_uint32)]


# Every symbol declared in include/*.h, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    # nomad_scene.h
    "nomad_scenebvh_build": (C.c_int32, [C.POINTER(SceneDesc), C.c_uint32, C.POINTER(_P)]),
    "nomad_scenebvh_build_gpu": (C.c_int32, [C.POINTER(SceneDesc), C.c_int32, C.POINTER(_P)]),
    "nomad_scenebvh_view_get": (C.c_int32, [_P, C.POINTER(SceneBVHView)]),
    "nomad_compact_workspace_bytes": (C.c_size_t, [C.c_uint32, C.c_uint32, C.c_uint32]),
    "nomad_scenebvh_compact_gpu": (C.c_int32, [C.POINTER(ScenebvhDevice), _P, _P, C.c_size_t,
                                               C.POINTER(CompactOut), _P]),
    "nomad_scenebvh_free": (None, [_P]),
    "nomad_synth_icospheres": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_float, C.POINTER(_P)]),
    "nomad_synth_city": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_uint32, C.c_float, C.c_uint32, C.c_uint32,
                                     C.c_uint32, C.c_uint32, C.c_uint32, C.c_float, C.POINTER(_P)]),
    "nomad_scene_owned_desc": (C.c_int32, [_P, C.POINTER(SceneDesc)]),
    "nomad_scene_owned_free": (None, [_P]),
    "nomad_scene_load_xml": (C.c_int32, [C.c_char_p, C.c_uint32, C.POINTER(_P)]),
    "nomad_loaded_scene_view_get": (C.c_int32, [_P, C.c_void_p]),
    "nomad_loaded_scene_free": (None, [_P]),
    "nomad_scene_last_error": (C.c_char_p, []),
    # nomad_rt.h
    "nomad_create": (C.c_int32, [C.POINTER(Config), C.POINTER(_P)]),
    "nomad_destroy": (C.c_int32, [_P]),
    "nomad_last_error": (C.c_char_p, [_P]),
    "nomad_sync": (C.c_int32, [_P]),
    "nomad_set_stream": (C.c_int32, [_P, _P]),
    "nomad_get_status": (C.c_int32, [_P, C.POINTER(C.c_uint32)]),
    "nomad_scene_upload": (C.c_int32, [_P, _P, C.c_uint32, _P, C.c_uint32, _P, _P, _P, C.c_uint32,
                                       _P, C.c_uint32]),
    "nomad_residency_set_primitive_active": (C.c_int32, [_P, C.c_uint32, C.c_int32,
                                                         C.POINTER(C.c_int32)]),
    "nomad_residency_set_object_active": (C.c_int32, [_P, C.c_uint32, C.c_int32,
                                                      C.POINTER(C.c_uint32)]),
    "nomad_residency_flush": (C.c_int32, [_P]),
    "nomad_residency_get_instances": (C.c_int32, [_P, _P]),
    "nomad_trace_closest": (C.c_int32, [_P, _P, C.c_uint64, _P, C.c_uint32]),
    "nomad_trace_any": (C.c_int32, [_P, _P, C.c_uint64, _P, C.c_uint32]),
    "nomad_set_kernel": (C.c_int32, [_P, C.c_uint32]),
    "nomad_trace_work": (C.c_int32, [_P, _P, C.c_uint64, _P, C.c_uint32]),
    "nomad_read_object_hits": (C.c_int32, [_P, _P]),
    "nomad_reset_object_hits": (C.c_int32, [_P]),
    "nomad_trace_closest_noalloc": (C.c_int32, [_P, _P, C.c_uint64, _P, _P]),
    "nomad_paging_enable": (C.c_int32, [_P, C.POINTER(PagingConfig)]),
    "nomad_paging_update": (C.c_int32, [_P]),
    "nomad_paging_wait": (C.c_int32, [_P]),
    "nomad_paging_set_sync": (C.c_int32, [_P, C.c_int32]),
    "nomad_paging_stats_get": (C.c_int32, [_P, C.POINTER(PagingStats)]),
    "nomad_paging_states": (C.c_int32, [_P, _P]),
    "nomad_view_pinhole": (C.c_int32, [_P, _P, _P, C.c_float, C.c_uint32, C.c_uint32, _P]),
    "nomad_render_frame": (C.c_int32, [_P, _P, C.c_uint32, _P, C.c_uint32]),
    "nomad_render_tiles": (C.c_int32, [_P, _P, _P, C.c_uint32, _P, C.c_uint32]),
    "nomad_render_stats": (C.c_int32, [_P, _P]),
    "nomad_frame_graph_stats": (C.c_int32, [_P, _P]),
    "nomad_reset_render_stats": (C.c_int32, [_P]),
    "nomad_residency_step": (C.c_int32, [_P, _P, _P, C.POINTER(C.c_uint32)]),
    "nomad_object_bytes": (C.c_int32, [_P, _P]),
    "nomad_residency_last": (C.c_int32, [_P, _P, _P]),
    "nomad_residency_flags": (C.c_int32, [_P, _P]),
    "nomad_residency_fallback_steps": (C.c_int32, [_P, C.POINTER(C.c_uint64)]),
    "nomad_selftest_bounded_wait": (C.c_int32, [_P, C.c_int32]),
    "nomad_residency_prim_state": (C.c_int32, [_P, _P, _P, _P, _P, _P]),
    "nomad_residency_object_state": (C.c_int32, [_P, _P, _P, _P]),
    "nomad_mlp_init": (C.c_int32, [_P, C.c_uint64]),
    "nomad_mlp_gradient": (C.c_int32, [_P, _P, _P, C.c_uint64, _P, _P]),
    "nomad_read_object_hits_ex": (C.c_int32, [_P, _P, C.c_uint32]),
    "nomad_write_object_hits": (C.c_int32, [_P, _P, C.c_uint32]),
    "nomad_residency_posterior": (C.c_int32, [_P, _P]),
    "nomad_residency_count_tests": (C.c_int32, [_P, C.c_int32, _P]),
    "nomad_mlp_train": (C.c_int32, [_P, _P, _P, C.c_uint64, C.c_uint32, C.c_uint32, C.c_float,
                                    C.c_float, C.c_uint64, _P]),
    "nomad_mlp_infer": (C.c_int32, [_P, _P, C.c_uint64, _P, C.c_uint32]),
    "nomad_mlp_get": (C.c_int32, [_P, _P]),
    "nomad_mlp_set": (C.c_int32, [_P, _P]),
    "nomad_mlp_save": (C.c_int32, [_P, C.c_char_p]),
    "nomad_mlp_load": (C.c_int32, [_P, C.c_char_p]),
    "nomad_set_restir": (C.c_int32, [_P, _P]),
    "nomad_reset_restir": (C.c_int32, [_P]),
    "nomad_autotune": (C.c_int32, [_P, _P, C.c_uint64, C.c_uint32, C.c_uint32, _P]),
    "nomad_set_traversal": (C.c_int32, [_P, _P]),
    "nomad_get_traversal": (C.c_int32, [_P, _P]),
    "nomad_tlas_nodes": (C.c_int32, [_P, _P]),
    "nomad_autotune_sweep": (C.c_int32, [_P, _P, C.c_uint64, C.c_uint32, C.c_uint32, _P, C.c_uint32,
                                         C.POINTER(C.c_uint32), _P]),
}

KERNEL_BVH4, KERNEL_BVH4_PERSIST, KERNEL_BVH8, KERNEL_BVH8_PERSIST, KERNEL_COUNT = 3, 4, 5, 6, 7
KERNEL_NAMES = {1: "bvh2", 2: "bvh2_persist", 3: "bvh4", 4: "bvh4_persist", 5: "bvh8", 6: "bvh8_persist"}


class TuneResult(C.Structure):
    _fields_ = [("best", C.c_uint32), ("ms", C.c_float * 7), ("mismatches", C.c_uint32 * 7),
                ("stack_need", C.c_uint32 * 3)]


class Traversal(C.Structure):
    """nomad_traversal: width, persistent (0, 1, 2 = regrouping), short_stack, regroup,
    staged_nodes, block, postpone_leaves."""
    _fields_ = [("width", C.c_uint32), ("persistent", C.c_uint32), ("short_stack", C.c_uint32),
                ("regroup", C.c_uint32), ("staged_nodes", C.c_uint32), ("block", C.c_uint32),
                ("postpone_leaves", C.c_uint32), ("min_blocks", C.c_uint32)]

    def as_dict(self) -> dict:
        return {f: int(getattr(self, f)) for f, _ in self._fields_}

    def name(self) -> str:
        if self.persistent == 3:
            return f"bvh{self.width}_packet"
        if self.persistent < 2:
            return (f"bvh{self.width}" + ("_persist" if self.persistent else "")
                    + (f"_mb{self.min_blocks}" if self.min_blocks else ""))
        return (f"bvh{self.width}_rg{self.regroup}_ss{self.short_stack}" + ("_post" if self.postpone_leaves else "")
                + (f"_st{self.staged_nodes}" if self.staged_nodes else "") + f"_b{self.block}")


class TuneEntry(C.Structure):
    _fields_ = [("cfg", Traversal), ("ms", C.c_float), ("mismatches", C.c_uint32)]


class RestirConfig(C.Structure):
    _fields_ = [("candidates", C.c_uint32), ("temporal", C.c_uint32), ("spatial", C.c_uint32),
                ("radius_px", C.c_float), ("m_cap", C.c_float), ("reference_mode", C.c_uint32)]

POLICY_ALWAYS, POLICY_RAYHIT_BUDGET, POLICY_LEARNED, POLICY_RAYHIT_PRIM, POLICY_DISTANCE_LOD = 0, 1, 2, 3, 4
POLICY_SCREEN_SPACE = 5
POLICY_PROBABILISTIC = 6
POLICY_ENVIRONMENT_HIT = 7
POLICY_PREDICTIVE = 8
POLICY_ENERGY = 9
N_FEATURES = 24
MLP_PARAMS = 128 * 32 + 128 + 128 * 128 + 128 + 128 + 1 + 2 * N_FEATURES


class ResidencyParams(C.Structure):
    _fields_ = [("policy", C.c_uint32), ("max_toggles", C.c_uint32), ("budget_bytes", C.c_uint64),
                ("hit_decay", C.c_float), ("camera_motion", C.c_float),
                ("memory_pressure", C.c_float), ("reserve_base", C.c_float),
                ("reserve_motion", C.c_float), ("min_active", C.c_uint32), ("target_fraction", C.c_float),
                ("rebuild_cooldown", C.c_uint32), ("state_cooldown", C.c_uint32),
                ("lod_enter_distance", C.c_float), ("lod_exit_distance", C.c_float),
                ("lod_enter_view_degrees", C.c_float), ("lod_exit_view_degrees", C.c_float),
                ("min_pixel_coverage", C.c_float),
                ("probability_decay", C.c_float), ("probability_window", C.c_float),
                ("probability_idle_frames", C.c_uint32), ("probability_idle_decay", C.c_float),
                ("probability_threshold", C.c_float), ("rayhit_prior_scale", C.c_float),
                ("uncertainty_boost", C.c_float), ("desired_hysteresis", C.c_float),
                ("visible_floor", C.c_float), ("recent_promotion_frames", C.c_uint32),
                ("demotion_dwell_frames", C.c_uint32), ("env_escape_threshold", C.c_float),
                ("env_high_escape", C.c_float), ("env_low_escape", C.c_float),
                ("energy_visibility_boost", C.c_float), ("energy_smoothing", C.c_float),
                ("energy_use_average", C.c_uint32), ("resident_key_bonus", C.c_float)]

    @staticmethod
    def make(policy, budget_bytes=0, max_toggles=0, hit_decay=0.85, camera_motion=0.0,
             memory_pressure=0.0, reserve_base=0.02, reserve_motion=0.06, min_active=0,
             target_fraction=0.54, rebuild_cooldown=4, state_cooldown=5, lod_enter_distance=225.0,
             lod_exit_distance=275.0, lod_enter_view_degrees=5.0, lod_exit_view_degrees=12.0,
             min_pixel_coverage=32.0, probability_decay=0.9, probability_window=64.0,
             probability_idle_frames=0, probability_idle_decay=0.9, probability_threshold=0.5,
             rayhit_prior_scale=0.0, uncertainty_boost=0.25, desired_hysteresis=0.02, visible_floor=0.0,
             recent_promotion_frames=4, demotion_dwell_frames=0, env_escape_threshold=0.4,
             env_high_escape=0.6, env_low_escape=0.3, energy_visibility_boost=1.75, energy_smoothing=0.85,
             energy_use_average=1, resident_key_bonus=0.0):
        return ResidencyParams(policy, max_toggles, budget_bytes, hit_decay, camera_motion,
                               memory_pressure, reserve_base, reserve_motion, min_active, target_fraction,
                               rebuild_cooldown, state_cooldown, lod_enter_distance, lod_exit_distance,
                               lod_enter_view_degrees, lod_exit_view_degrees, min_pixel_coverage,
                               probability_decay, probability_window, probability_idle_frames,
                               probability_idle_decay, probability_threshold, rayhit_prior_scale,
                               uncertainty_boost, desired_hysteresis, visible_floor, recent_promotion_frames,
                               demotion_dwell_frames, env_escape_threshold, env_high_escape, env_low_escape,
                               energy_visibility_boost, energy_smoothing, energy_use_average,
                               resident_key_bonus)

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}

VIEW_DTYPE = np.dtype([("camera_pos", "<f4", 3), ("viewport_u", "<f4", 3), ("viewport_v", "<f4", 3),
                       ("first_pixel", "<f4", 3), ("width", "<u4"), ("height", "<u4"), ("spp", "<u4"),
                       ("max_depth", "<u4"), ("seed_lo", "<u4"), ("seed_hi", "<u4"), ("frame", "<u4"),
                       ("flags", "<u4")])
VIEW_CLAMP = 1 << 0
VIEW_RESTIR = 1 << 1
VIEW_CENTER = 1 << 2
RENDER_DIRECT = 1 << 2  # render flag: launch the frame without the cached CUDA graph


def view_pinhole(position, look_at, up=(0.0, 1.0, 0.0), vfov=60.0, width=640, height=360, spp=1,
                 max_depth=1, seed=0, frame=0, flags=0) -> np.ndarray:
    """A nomad_view (numpy record) for a pinhole camera, filled by the library
    (populateViewportUniforms semantics)."""
    lib = load()
    out = np.zeros(1, VIEW_DTYPE)
    pos = np.asarray(position, np.float32)
    look = np.asarray(look_at, np.float32)
    upv = np.asarray(up, np.float32)
    _check(lib.nomad_view_pinhole(pos.ctypes.data, look.ctypes.data, upv.ctypes.data, vfov, width,
                                  height, out.ctypes.data))
    out["spp"], out["max_depth"], out["frame"], out["flags"] = spp, max_depth, frame, flags
    out["seed_lo"], out["seed_hi"] = seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF
    return out

_lib: Optional[C.CDLL] = None


def load() -> C.CDLL:
    """Loads libnomad_rt.so; raises when it is missing (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C nomad_b200/csrc`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _ptr(a) -> int:
    """Address of a contiguous numpy array or a torch tensor."""
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


# ---------------------------------------------------------------------------------------------
# Host scenes


class HostScene:
    """A scene description (primitives grouped into objects) as numpy arrays."""

    def __init__(self, prim_type, prim_geom, prim_material, object_first, object_prims):
        self.prim_type = np.ascontiguousarray(prim_type, dtype=np.int32)
        self.prim_geom = _f(prim_geom).reshape(-1, 15)
        self.prim_material = _f(prim_material).reshape(-1, 20)
        self.object_first = np.ascontiguousarray(object_first, dtype=np.uint32)
        self.object_prims = np.ascontiguousarray(object_prims, dtype=np.uint32)

    @property
    def prim_count(self) -> int:
        return int(self.prim_type.shape[0])

    @property
    def object_count(self) -> int:
        return int(self.object_first.shape[0])

    def desc(self) -> SceneDesc:
        d = SceneDesc()
        d.prim_count = self.prim_count
        d.prim_type = self.prim_type.ctypes.data_as(C.POINTER(C.c_int32))
        d.prim_geom = self.prim_geom.ctypes.data_as(C.POINTER(C.c_float))
        d.prim_material = self.prim_material.ctypes.data_as(C.POINTER(C.c_float))
        d.object_count = self.object_count
        d.object_first = self.object_first.ctypes.data_as(C.POINTER(C.c_uint32))
        d.object_prims = self.object_prims.ctypes.data_as(C.POINTER(C.c_uint32))
        return d

    @staticmethod
    def _from_owned(h) -> "HostScene":
        lib = load()
        d = SceneDesc()
        _check(lib.nomad_scene_owned_desc(h, C.byref(d)))
        n, m = d.prim_count, d.object_count
        s = HostScene(np.ctypeslib.as_array(d.prim_type, (n,)).copy(),
                      np.ctypeslib.as_array(d.prim_geom, (n * 15,)).copy(),
                      np.ctypeslib.as_array(d.prim_material, (n * 20,)).copy(),
                      np.ctypeslib.as_array(d.object_first, (m,)).copy(),
                      np.ctypeslib.as_array(d.object_prims, (m,)).copy())
        lib.nomad_scene_owned_free(h)
        return s


class LoadedScene(HostScene):
    """A scene read from the reference's XML format (nomad_scene_load_xml): the scene description
    plus each object's mesh group, the root's settings, the camera path and the observer camera."""

    def __init__(self, path: str, threads: int = 0):
        lib = load()
        h = _P()
        st = lib.nomad_scene_load_xml(os.fsencode(path), threads, C.byref(h))
        if st != NOMAD_OK:
            raise NomadError(st, (lib.nomad_scene_last_error() or b"").decode())
        try:
            v = LoadedSceneView()
            _check(lib.nomad_loaded_scene_view_get(h, C.byref(v)))
            d = v.scene
            n, m = d.prim_count, d.object_count

            def arr(ptr, count, dtype):
                return np.ctypeslib.as_array(ptr, (count,)).copy() if count else np.zeros(0, dtype)

            super().__init__(arr(d.prim_type, n, np.int32), arr(d.prim_geom, n * 15, np.float32),
                             arr(d.prim_material, n * 20, np.float32), arr(d.object_first, m, np.uint32),
                             arr(d.object_prims, m, np.uint32))
            self.object_mesh_group = arr(v.object_mesh_group, m, np.int32)
            self.settings = v.settings.as_dict()
            self.keyframes = [
                {"frame": k.frame, "position": tuple(k.position), "look_at": tuple(k.look_at), "up": tuple(k.up),
                 "aperture": k.aperture, "focus_distance": k.focus_distance}
                for k in (v.keyframes[i] for i in range(v.keyframe_count))]
            o = v.observer
            self.observer = ({"position": tuple(o.position), "look_at": tuple(o.look_at), "up": tuple(o.up),
                              "vertical_fov": o.vertical_fov, "aperture": o.aperture,
                              "focus_distance": o.focus_distance} if v.has_observer else None)
            self.environment_texture = (v.environment_texture or b"").decode()
            self.mesh_files, self.mesh_files_failed = v.mesh_files, v.mesh_files_failed
            self.log = (v.log or b"").decode()
        finally:
            lib.nomad_loaded_scene_free(h)


def load_scene_xml(path: str, threads: int = 0) -> LoadedScene:
    """Reads a scene XML with its OBJ/MTL meshes (the reference's SceneLoader format)."""
    return LoadedScene(path, threads)


def synth_icospheres(seed: int, instances: int = 64, extent: float = 100.0) -> HostScene:
    lib = load()
    h = _P()
    _check(lib.nomad_synth_icospheres(seed, instances, extent, C.byref(h)))
    return HostScene._from_owned(h)


def synth_city(seed: int, grid: int = 32, size_m: float = 1000.0, target_tris: int = 2_500_000,
               median_tris: int = 1000, max_tris: int = 200_000, emissive_quads: int = 64,
               emissive_tris: int = 0, emissive_sigma: float = 1.5, grid_z: int = 0) -> HostScene:
    lib = load()
    h = _P()
    _check(lib.nomad_synth_city(seed, grid, grid_z or grid, size_m, target_tris, median_tris, max_tris,
                                emissive_quads, emissive_tris, emissive_sigma, C.byref(h)))
    return HostScene._from_owned(h)


class SceneBVH:
    """SceneBVH arrays (reference GPU layouts) built from a HostScene, as numpy copies."""

    def __init__(self, scene: HostScene, threads: int = 0, device: int | None = None):
        """Builds on host threads, or with the per-object BLAS builds on CUDA device `device`
        (the same arrays, bit for bit)."""
        lib = load()
        h = _P()
        d = scene.desc()
        if device is None:
            _check(lib.nomad_scenebvh_build(C.byref(d), threads, C.byref(h)))
        else:
            _check(lib.nomad_scenebvh_build_gpu(C.byref(d), device, C.byref(h)))
        try:
            v = SceneBVHView()
            _check(lib.nomad_scenebvh_view_get(h, C.byref(v)))
            self.prim_count = v.prim_count
            self.object_count = v.object_count
            self.bvh_nodes = np.ctypeslib.as_array(v.bvh_nodes, (v.bvh_node_count * 8,)).copy()
            self.tlas_nodes = np.ctypeslib.as_array(v.tlas_nodes, (v.tlas_node_count * 8,)).copy()
            self.prims = np.ctypeslib.as_array(v.prims, (v.prim_count * 28,)).copy()
            self.materials = np.ctypeslib.as_array(v.materials, (v.prim_count * 20,)).copy()
            self.prim_indices = np.ctypeslib.as_array(v.prim_indices, (v.prim_count,)).copy()
            inst = (C.c_char * (v.object_count * 16)).from_address(v.instances)
            self.instances = np.frombuffer(bytes(inst), dtype=INSTANCE_DTYPE).copy()
            self.object_bounds = np.ctypeslib.as_array(v.object_bounds, (v.object_count * 6,)).copy()
            self.max_depth = v.max_depth
        finally:
            lib.nomad_scenebvh_free(h)
        self.prim_object = np.repeat(np.arange(self.object_count, dtype=np.int32),
                                     self.instances["primitive_count"].astype(np.int64))

    @property
    def bvh_node_count(self) -> int:
        return self.bvh_nodes.size // 8

    @property
    def tlas_node_count(self) -> int:
        return self.tlas_nodes.size // 8

    def geometry_bytes_per_object(self) -> np.ndarray:
        """Bytes an object occupies on the device: 32 per BLAS node plus 112 + 80 + 4 per
        primitive (packed primitive, material, index)."""
        nodes = np.zeros(self.object_count, np.int64)
        # Node blocks are per object and in object order: count them via the roots.
        roots = self.instances["blas_root_index"].astype(np.int64)
        order = np.argsort(roots)
        bounds = np.append(roots[order], self.bvh_node_count)
        nodes[order] = np.diff(bounds)
        return 32 * nodes + 196 * self.instances["primitive_count"].astype(np.int64)


class Compactor:
    """Residency compaction on the device (nomad_scenebvh_compact_gpu) of one SceneBVH, uploaded
    once; outputs stay in device memory (torch tensors) until result() copies them back."""

    def __init__(self, sb: SceneBVH, device: str = "cuda:0"):
        import torch
        self._torch = torch
        lib = load()

        def up(a):
            return torch.from_numpy(np.ascontiguousarray(a)).to(device)

        n, nn, nobj = int(sb.prim_count), int(sb.bvh_node_count), int(sb.object_count)
        self.sizes = (n, nn, nobj)
        self.bvh, self.prims, self.mats = up(sb.bvh_nodes), up(sb.prims), up(sb.materials)
        self.idx = up(sb.prim_indices)
        self.inst = up(sb.instances.view(np.int32).reshape(-1))
        self.inp = ScenebvhDevice(n, nobj, nn, 0, self.bvh.data_ptr(), self.prims.data_ptr(),
                                  self.mats.data_ptr(), self.idx.data_ptr(), self.inst.data_ptr())
        self.ws_bytes = int(lib.nomad_compact_workspace_bytes(n, nn, nobj))
        self.ws = torch.empty(self.ws_bytes, dtype=torch.uint8, device=device)
        f32, i32 = torch.float32, torch.int32
        self.o_bvh = torch.empty(max(nn, 1) * 8, dtype=f32, device=device)
        self.o_prims = torch.empty(n * 28, dtype=f32, device=device)
        self.o_mats = torch.empty(n * 20, dtype=f32, device=device)
        self.o_idx = torch.empty(n, dtype=i32, device=device)
        self.o_remap = torch.empty(n, dtype=i32, device=device)
        self.o_p2r = torch.empty(n, dtype=i32, device=device)
        self.o_inst = torch.empty(nobj * 4, dtype=i32, device=device)
        self.o_counts = torch.zeros(3, dtype=i32, device=device)
        self.out = CompactOut(self.o_bvh.data_ptr(), self.o_prims.data_ptr(), self.o_mats.data_ptr(),
                              self.o_idx.data_ptr(), self.o_remap.data_ptr(), self.o_p2r.data_ptr(),
                              self.o_inst.data_ptr(), self.o_counts.data_ptr())

    def run(self, active) -> None:
        """Queues one compaction for the per-primitive mask `active` (a uint8 device tensor, or a
        host array uploaded first) on torch's current stream."""
        torch = self._torch
        if not isinstance(active, torch.Tensor):
            active = torch.from_numpy(np.ascontiguousarray(active, np.uint8)).to(self.bvh.device)
        assert active.dtype == torch.uint8 and active.numel() == self.sizes[0]
        self._active = active
        stream = torch.cuda.current_stream(self.bvh.device).cuda_stream
        _check(load().nomad_scenebvh_compact_gpu(C.byref(self.inp), active.data_ptr(), self.ws.data_ptr(),
                                                 self.ws_bytes, C.byref(self.out), stream))

    def result(self) -> dict:
        """The last compaction's arrays, trimmed to their lengths, as numpy (synchronises)."""
        counts = self.o_counts.cpu().numpy().astype(np.uint32)
        if counts[2]:
            raise NomadError(5, f"compaction error bits {int(counts[2])}")
        p, nodes = int(counts[0]), int(counts[1])
        return {
            "prim_count": p, "bvh_node_count": nodes,
            "bvh_nodes": self.o_bvh[: nodes * 8].cpu().numpy(),
            "prims": self.o_prims[: p * 28].cpu().numpy(),
            "materials": self.o_mats[: p * 20].cpu().numpy(),
            "prim_indices": self.o_idx[:p].cpu().numpy(),
            "remap": self.o_remap[:p].cpu().numpy().view(np.uint32),
            "prim_to_resident": self.o_p2r.cpu().numpy(),
            "instances": self.o_inst.cpu().numpy().view(INSTANCE_DTYPE),
        }


def _check(st: int, ctx=None):
    if st != NOMAD_OK:
        msg = ""
        if ctx is not None:
            m = load().nomad_last_error(ctx)
            msg = m.decode() if m else ""
        raise NomadError(st, msg)


# ---------------------------------------------------------------------------------------------
# Device context


class Context:
    """One libnomad_rt context on one CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load()
        cfg = Config(device, 0)
        h = _P()
        _check(self.lib.nomad_create(C.byref(cfg), C.byref(h)))
        self.h = h
        self.object_count = 0
        self.prim_count = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.nomad_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, st):
        _check(st, self.h)

    def upload(self, s: SceneBVH, instances: Optional[np.ndarray] = None):
        inst = s.instances if instances is None else np.ascontiguousarray(instances, INSTANCE_DTYPE)
        self._keep = (s, inst)
        self._ck(self.lib.nomad_scene_upload(
            self.h, _ptr(s.bvh_nodes), s.bvh_node_count, _ptr(s.tlas_nodes), s.tlas_node_count,
            _ptr(s.prims), _ptr(s.materials), _ptr(s.prim_indices), s.prim_count, _ptr(inst),
            s.object_count))
        self.object_count = s.object_count
        self.prim_count = s.prim_count

    def set_stream(self, stream_handle: int):
        self._ck(self.lib.nomad_set_stream(self.h, _P(stream_handle) if stream_handle else None))

    def autotune(self, rays, repeats=3, device=False) -> dict:
        """Times every traversal variant on the sample rays (numpy records, or a device pointer
        with device=True and rays=(ptr, n)), selects the fastest; returns the table."""
        r = TuneResult()
        if device:
            ptr, n = rays
            self._ck(self.lib.nomad_autotune(self.h, _P(ptr), n, repeats, TRACE_DEVICE_POINTERS, C.byref(r)))
        else:
            rr = np.ascontiguousarray(rays, RAY_DTYPE)
            self._ck(self.lib.nomad_autotune(self.h, _ptr(rr), rr.shape[0], repeats, 0, C.byref(r)))
        return {"best": KERNEL_NAMES.get(r.best, str(r.best)), "best_id": int(r.best),
                "ms": {KERNEL_NAMES[k]: float(r.ms[k]) for k in range(1, 7)},
                "mismatches": {KERNEL_NAMES[k]: int(r.mismatches[k]) for k in range(1, 7)},
                "stack_need": list(r.stack_need)}

    def set_kernel(self, k: int):
        self._ck(self.lib.nomad_set_kernel(self.h, k))

    def set_traversal(self, width=2, persistent=2, short_stack=0, regroup=1, staged_nodes=0, block=128,
                      postpone_leaves=0, min_blocks=0):
        t = Traversal(width, persistent, short_stack, regroup, staged_nodes, block, postpone_leaves, min_blocks)
        self._ck(self.lib.nomad_set_traversal(self.h, C.byref(t)))

    def traversal(self) -> dict:
        t = Traversal()
        self._ck(self.lib.nomad_get_traversal(self.h, C.byref(t)))
        return t.as_dict()

    def tlas_nodes(self) -> list:
        out = (C.c_uint32 * 3)()
        self._ck(self.lib.nomad_tlas_nodes(self.h, out))
        return list(out)

    def autotune_sweep(self, rays, repeats=2, device=False) -> dict:
        """Sweeps width x short stack x regroup threshold x staged top levels x block on the sample
        rays, checks each configuration bit for bit against the binary kernel and selects the
        fastest; returns {"best": cfg dict, "best_name", "entries": [(name, cfg, ms, mismatches)]}."""
        cap = 1024
        entries = (TuneEntry * cap)()
        count = C.c_uint32(0)
        best = Traversal()
        if device:
            ptr, n = rays
            self._ck(self.lib.nomad_autotune_sweep(self.h, _P(ptr), n, repeats, TRACE_DEVICE_POINTERS, entries, cap,
                                                   C.byref(count), C.byref(best)))
        else:
            rr = np.ascontiguousarray(rays, RAY_DTYPE)
            self._ck(self.lib.nomad_autotune_sweep(self.h, _ptr(rr), rr.shape[0], repeats, 0, entries, cap,
                                                   C.byref(count), C.byref(best)))
        rows = [(e.cfg.name(), e.cfg.as_dict(), float(e.ms), int(e.mismatches))
                for e in entries[: min(count.value, cap)]]
        return {"best": best.as_dict(), "best_name": best.name(), "entries": rows}

    def sync(self):
        self._ck(self.lib.nomad_sync(self.h))

    def status(self) -> int:
        w = C.c_uint32()
        self._ck(self.lib.nomad_get_status(self.h, C.byref(w)))
        return w.value

    # residency
    def set_object_active(self, obj: int, active: bool) -> int:
        t = C.c_uint32()
        self._ck(self.lib.nomad_residency_set_object_active(self.h, obj, int(active), C.byref(t)))
        return t.value

    def set_primitive_active(self, prim: int, active: bool) -> bool:
        c = C.c_int32()
        self._ck(self.lib.nomad_residency_set_primitive_active(self.h, prim, int(active), C.byref(c)))
        return bool(c.value)

    def flush(self):
        self._ck(self.lib.nomad_residency_flush(self.h))

    def instances(self) -> np.ndarray:
        out = np.zeros(self.object_count, INSTANCE_DTYPE)
        self._ck(self.lib.nomad_residency_get_instances(self.h, _ptr(out)))
        return out

    # traversal (host arrays)
    def trace_closest(self, rays: np.ndarray, count_hits: bool = False) -> np.ndarray:
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.empty(rays.shape[0], HIT_DTYPE)
        self._ck(self.lib.nomad_trace_closest(self.h, _ptr(rays), rays.shape[0], _ptr(out),
                                              TRACE_COUNT_HITS if count_hits else 0))
        return out

    def trace_any(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.empty(rays.shape[0], np.uint8)
        self._ck(self.lib.nomad_trace_any(self.h, _ptr(rays), rays.shape[0], _ptr(out), 0))
        return out

    def trace_work(self, rays: np.ndarray) -> np.ndarray:
        rays = np.ascontiguousarray(rays, RAY_DTYPE)
        out = np.empty((rays.shape[0], 4), np.uint32)
        self._ck(self.lib.nomad_trace_work(self.h, _ptr(rays), rays.shape[0], _ptr(out), 0))
        return out

    # traversal (device pointers, e.g. torch tensors); asynchronous on the context stream
    def trace_closest_dev(self, rays_ptr: int, n: int, hits_ptr: int, count_hits: bool = False):
        self._ck(self.lib.nomad_trace_closest(self.h, _P(rays_ptr), n, _P(hits_ptr),
                                              TRACE_DEVICE_POINTERS |
                                              (TRACE_COUNT_HITS if count_hits else 0)))

    def trace_any_dev(self, rays_ptr: int, n: int, out_ptr: int):
        self._ck(self.lib.nomad_trace_any(self.h, _P(rays_ptr), n, _P(out_ptr),
                                          TRACE_DEVICE_POINTERS))

    def trace_work_dev(self, rays_ptr: int, n: int, out_ptr: int):
        self._ck(self.lib.nomad_trace_work(self.h, _P(rays_ptr), n, _P(out_ptr),
                                           TRACE_DEVICE_POINTERS))

    # path tracing
    def render(self, views: np.ndarray, count_hits: bool = False, graph: bool = True) -> list:
        """Renders the views in one batched frame (replayed from a captured CUDA graph unless
        graph=False); returns one (height, width, 3) float32 image per view."""
        views = np.ascontiguousarray(views, VIEW_DTYPE).reshape(-1)
        total = int((views["width"].astype(np.int64) * views["height"]).sum())
        out = np.empty(total * 3, np.float32)
        flags = (TRACE_COUNT_HITS if count_hits else 0) | (0 if graph else RENDER_DIRECT)
        self._ck(self.lib.nomad_render_frame(self.h, _ptr(views), views.shape[0], _ptr(out), flags))
        imgs, off = [], 0
        for v in views:
            n = int(v["width"]) * int(v["height"])
            imgs.append(out[3 * off:3 * (off + n)].reshape(int(v["height"]), int(v["width"]), 3))
            off += n
        return imgs

    def render_dev(self, views: np.ndarray, out_ptr: int, count_hits: bool = False, graph: bool = True):
        views = np.ascontiguousarray(views, VIEW_DTYPE).reshape(-1)
        self._keep_views = views
        self._ck(self.lib.nomad_render_frame(self.h, _ptr(views), views.shape[0], _P(out_ptr),
                                             TRACE_DEVICE_POINTERS |
                                             (TRACE_COUNT_HITS if count_hits else 0) |
                                             (0 if graph else RENDER_DIRECT)))

    def render_tiles(self, views: np.ndarray, tiles, count_hits: bool = False, graph: bool = True) -> list:
        """Renders tiles[i] = (origin_x, origin_y, width, height) of views[i] in one batched frame;
        returns one (height, width, 3) float32 image per tile, equal bit for bit to that region
        of render() of the same views."""
        views = np.ascontiguousarray(views, VIEW_DTYPE).reshape(-1)
        tiles = np.ascontiguousarray(np.asarray(tiles, np.uint32).reshape(-1, 4))
        if tiles.shape[0] != views.shape[0]:
            raise ValueError("one tile per view")
        total = int((tiles[:, 2].astype(np.int64) * tiles[:, 3]).sum())
        out = np.empty(total * 3, np.float32)
        flags = (TRACE_COUNT_HITS if count_hits else 0) | (0 if graph else RENDER_DIRECT)
        self._ck(self.lib.nomad_render_tiles(self.h, _ptr(views), _ptr(tiles), views.shape[0], _ptr(out), flags))
        imgs, off = [], 0
        for t in tiles:
            n = int(t[2]) * int(t[3])
            imgs.append(out[3 * off:3 * (off + n)].reshape(int(t[3]), int(t[2]), 3))
            off += n
        return imgs

    def render_tiles_dev(self, views: np.ndarray, tiles, out_ptr: int, count_hits: bool = False,
                         graph: bool = True):
        """render_tiles into device memory at out_ptr (the tiles' pixels, 3 floats each)."""
        views = np.ascontiguousarray(views, VIEW_DTYPE).reshape(-1)
        tiles = np.ascontiguousarray(np.asarray(tiles, np.uint32).reshape(-1, 4))
        if tiles.shape[0] != views.shape[0]:
            raise ValueError("one tile per view")
        self._keep_views = (views, tiles)
        self._ck(self.lib.nomad_render_tiles(self.h, _ptr(views), _ptr(tiles), views.shape[0], _P(out_ptr),
                                             TRACE_DEVICE_POINTERS |
                                             (TRACE_COUNT_HITS if count_hits else 0) |
                                             (0 if graph else RENDER_DIRECT)))

    def frame_graph_stats(self) -> dict:
        out = np.zeros(3, np.uint64)
        self._ck(self.lib.nomad_frame_graph_stats(self.h, _ptr(out)))
        return {"captures": int(out[0]), "launches": int(out[1]), "cached": int(out[2])}

    def render_stats(self) -> np.ndarray:
        out = np.zeros(4, np.uint64)
        self._ck(self.lib.nomad_render_stats(self.h, _ptr(out)))
        return out

    def reset_render_stats(self):
        self._ck(self.lib.nomad_reset_render_stats(self.h))

    # residency policies
    def residency_step(self, params: "ResidencyParams", camera_view: np.ndarray, toggles: bool = True):
        """One device residency step. With toggles=True waits for and returns the number of
        objects whose residency flipped; with toggles=False the step stays asynchronous on the
        context's stream (returns None)."""
        v = np.ascontiguousarray(camera_view, VIEW_DTYPE).reshape(-1)[:1]
        if not toggles:
            self._ck(self.lib.nomad_residency_step(self.h, C.byref(params), _ptr(v), None))
            return None
        t = C.c_uint32()
        self._ck(self.lib.nomad_residency_step(self.h, C.byref(params), _ptr(v), C.byref(t)))
        return t.value

    def object_bytes(self) -> np.ndarray:
        out = np.zeros(self.object_count, np.uint64)
        self._ck(self.lib.nomad_object_bytes(self.h, _ptr(out)))
        return out

    def residency_last(self):
        f = np.zeros((self.object_count, N_FEATURES), np.float32)
        s = np.zeros(self.object_count, np.float32)
        self._ck(self.lib.nomad_residency_last(self.h, _ptr(f), _ptr(s)))
        return f, s

    def residency_prim_state(self):
        """(hits since the last step, decayed scores, cooldowns, frustum test of the last step,
        activity) per primitive."""
        h = np.zeros(self.prim_count, np.uint32)
        sc = np.zeros(self.prim_count, np.float32)
        cd = np.zeros(self.prim_count, np.uint32)
        vis = np.zeros(self.prim_count, np.uint8)
        act = np.zeros(self.prim_count, np.uint8)
        self._ck(self.lib.nomad_residency_prim_state(self.h, _ptr(h), _ptr(sc), _ptr(cd), _ptr(vis), _ptr(act)))
        return h, sc, cd, vis, act

    def residency_object_state(self):
        """DistanceLOD state of the last step: (distance, flags 1 enter / 2 exit / 4 behind,
        cooldowns) per object."""
        d = np.zeros(self.object_count, np.float32)
        f = np.zeros(self.object_count, np.uint8)
        c = np.zeros(self.object_count, np.uint32)
        self._ck(self.lib.nomad_residency_object_state(self.h, _ptr(d), _ptr(f), _ptr(c)))
        return d, f, c

    def residency_posterior(self) -> dict:
        """The per-object hit-probability posterior after the last step."""
        out = np.zeros((self.object_count, 9), np.float32)
        self._ck(self.lib.nomad_residency_posterior(self.h, _ptr(out)))
        u = out.view(np.uint32)
        return {"alpha": out[:, 0].copy(), "beta": out[:, 1].copy(), "probability": out[:, 2].copy(),
                "variance": out[:, 3].copy(), "mass": out[:, 4].copy(), "exploration": out[:, 5].copy(),
                "idle": u[:, 6].copy(), "hits": u[:, 7].copy(), "tests": u[:, 8].copy()}

    def count_object_tests(self, on: bool = True, read: bool = False):
        """Switches per-object rays-tested counting on or off; with read, returns and clears the
        counts gathered since the last step or read."""
        out = np.zeros(self.object_count, np.uint32) if read else None
        self._ck(self.lib.nomad_residency_count_tests(self.h, 1 if on else 0, _ptr(out) if read else None))
        return out

    def residency_flags(self) -> np.ndarray:
        out = np.zeros(self.object_count, np.uint8)
        self._ck(self.lib.nomad_residency_flags(self.h, _ptr(out)))
        return out

    def selftest_bounded_wait(self, complete: bool):
        """Runs the bounded-wait self-test; read the outcome with status()."""
        self._ck(self.lib.nomad_selftest_bounded_wait(self.h, 1 if complete else 0))

    def residency_fallback_steps(self) -> int:
        """Learned-policy steps that ran the ray-hit budget for want of a usable model."""
        out = C.c_uint64()
        self._ck(self.lib.nomad_residency_fallback_steps(self.h, C.byref(out)))
        return int(out.value)

    # learned scorer
    def mlp_init(self, seed: int = 0):
        self._ck(self.lib.nomad_mlp_init(self.h, seed))

    def mlp_train(self, features, targets, steps=500, batch=1024, lr=1e-3, weight_decay=1e-4,
                  seed=0) -> np.ndarray:
        x = np.ascontiguousarray(features, np.float32)
        t = np.ascontiguousarray(targets, np.float32)
        loss = np.zeros(steps, np.float32)
        self._ck(self.lib.nomad_mlp_train(self.h, _ptr(x), _ptr(t), t.shape[0], steps, batch, lr,
                                          weight_decay, seed, _ptr(loss)))
        return loss

    def mlp_gradient(self, features, targets):
        """(gradient blob, mean squared error) of the current model over the samples in order."""
        x = np.ascontiguousarray(features, np.float32).reshape(-1, N_FEATURES)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = np.zeros(1, np.float32)
        self._ck(self.lib.nomad_mlp_gradient(self.h, _ptr(x), _ptr(t), t.shape[0], _ptr(g), _ptr(loss)))
        return g, float(loss[0])

    def mlp_infer(self, features) -> np.ndarray:
        x = np.ascontiguousarray(features, np.float32)
        out = np.zeros(x.shape[0], np.float32)
        self._ck(self.lib.nomad_mlp_infer(self.h, _ptr(x), x.shape[0], _ptr(out), 0))
        return out

    def mlp_get(self) -> np.ndarray:
        out = np.zeros(MLP_PARAMS, np.float32)
        self._ck(self.lib.nomad_mlp_get(self.h, _ptr(out)))
        return out

    def mlp_set(self, blob):
        b = np.ascontiguousarray(blob, np.float32)
        assert b.size == MLP_PARAMS
        self._ck(self.lib.nomad_mlp_set(self.h, _ptr(b)))

    def mlp_save(self, path: str):
        """Writes the model as a versioned, checksummed file."""
        self._ck(self.lib.nomad_mlp_save(self.h, os.fsencode(path)))

    def mlp_load(self, path: str):
        """Reads a model file; a bad file raises and leaves the context without a usable model
        (learned steps then run the ray-hit budget)."""
        self._ck(self.lib.nomad_mlp_load(self.h, os.fsencode(path)))

    # ReSTIR DI
    def set_restir(self, candidates=32, temporal=True, spatial=3, radius_px=30.0, m_cap=20.0,
                   reference_mode=False):
        cfg = RestirConfig(candidates, int(temporal), spatial, radius_px, m_cap, int(reference_mode))
        self._ck(self.lib.nomad_set_restir(self.h, C.byref(cfg)))

    def reset_restir(self):
        self._ck(self.lib.nomad_reset_restir(self.h))

    def object_hits(self) -> np.ndarray:
        out = np.zeros(self.object_count, np.uint32)
        self._ck(self.lib.nomad_read_object_hits(self.h, _ptr(out)))
        return out

    def object_hits_dev(self, out_ptr: int):
        """The per-object hit counts into a device array of object_count u32 words (queued on the
        context's stream)."""
        self._ck(self.lib.nomad_read_object_hits_ex(self.h, _P(out_ptr), TRACE_DEVICE_POINTERS))

    def write_object_hits(self, counts=None, dev_ptr: int = 0):
        """Replaces the hit counts gathered since the last residency step: a host array of
        object_count u32, or a device array (dev_ptr) queued on the context's stream."""
        if dev_ptr:
            self._ck(self.lib.nomad_write_object_hits(self.h, _P(dev_ptr), TRACE_DEVICE_POINTERS))
        else:
            c = np.ascontiguousarray(counts, np.uint32)
            assert c.size == self.object_count
            self._ck(self.lib.nomad_write_object_hits(self.h, _ptr(c), 0))

    # geometry paging
    def paging_enable(self, pool_bytes: int, width: int = 4, max_onloads: int = 0):
        cfg = PagingConfig(int(pool_bytes), int(max_onloads), int(width))
        self._ck(self.lib.nomad_paging_enable(self.h, C.byref(cfg)))

    def paging_update(self):
        self._ck(self.lib.nomad_paging_update(self.h))

    def paging_wait(self):
        self._ck(self.lib.nomad_paging_wait(self.h))

    def paging_set_sync(self, on: bool = True):
        """Updates wait for the previous updates' copies and releases, so runs repeat exactly."""
        self._ck(self.lib.nomad_paging_set_sync(self.h, 1 if on else 0))

    def paging_stats(self) -> dict:
        st = PagingStats()
        self._ck(self.lib.nomad_paging_stats_get(self.h, C.byref(st)))
        return {f: int(getattr(st, f)) for f, _ in PagingStats._fields_}

    def paging_states(self) -> np.ndarray:
        out = np.zeros(self.object_count, np.uint8)
        self._ck(self.lib.nomad_paging_states(self.h, _ptr(out)))
        return out

    def reset_object_hits(self):
        self._ck(self.lib.nomad_reset_object_hits(self.h))
