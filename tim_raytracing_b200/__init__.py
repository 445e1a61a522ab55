"""tim_raytracing_b200 -- B200 (sm_100a) implementation of TIM_Raytracing's
BVH traversal hot path behind a C ABI (include/tim_rt.h, libtim_rt.so).

The package holds the CUDA kernels and host runtime (csrc/), the in-tree build
(build.py), the ctypes binding of the ABI (_native.py) and the seeded
synthetic workloads (scenes.py).
"""
from . import scenes  # noqa: F401
from ._native import (  # noqa: F401
    BvhImage, Context, TimRtError, build_bvh, lib, validate,
    MODE_CLOSEST, MODE_ANY, MODE_PER_RAY, TRACE_WIDE, UPLOAD_QUANT8,
    CAM_PROB_MASK, CAM_TILE_LIGHTS, CAM_BOUNCE, CAM_WIDE,
)
