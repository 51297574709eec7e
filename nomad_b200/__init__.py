"""nomad_b200 — B200-native ray traversal / path-tracing core.

The compute path is libnomad_rt.so (hand-written sm_100a CUDA + host C++), reached through the
C ABI in include/nomad_rt.h and include/nomad_scene.h. This package only binds it (ctypes) and
builds host-side ray batches; it has no CPU fallback.
"""
from .native import (  # noqa: F401
    VIEW_DTYPE, VIEW_CLAMP, VIEW_RESTIR, VIEW_CENTER, view_pinhole, ResidencyParams, N_FEATURES, MLP_PARAMS,
    POLICY_ALWAYS, POLICY_RAYHIT_BUDGET, POLICY_LEARNED, POLICY_RAYHIT_PRIM, POLICY_DISTANCE_LOD,
    POLICY_SCREEN_SPACE, POLICY_PROBABILISTIC, POLICY_ENVIRONMENT_HIT, POLICY_PREDICTIVE, POLICY_ENERGY,
    RestirConfig,
    Context, HostScene, LoadedScene, SceneBVH, NomadError, load, load_scene_xml, synth_city, synth_icospheres,
    RAY_DTYPE, HIT_DTYPE, INSTANCE_DTYPE, LIB_PATH, SIGNATURES,
    KERNEL_AUTO, KERNEL_BVH2, KERNEL_BVH2_PERSIST, KERNEL_BVH4, KERNEL_BVH4_PERSIST, KERNEL_BVH8,
    KERNEL_BVH8_PERSIST, KERNEL_NAMES, TRACE_COUNT_HITS, TRACE_DEVICE_POINTERS,
)
from .rays import Camera, bounce_rays, city_camera, icosphere_camera, shadow_rays  # noqa: F401
