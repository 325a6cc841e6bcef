"""luvas3d: B200-native dense reconstruction (PatchMatch MVS + TSDF integration).

The Python side mirrors the scanner's stage API (DenseStereo, STEREO_METHODS, BrickGrid,
TsdfVolume) over the C ABI of libluvas3d.so; all device work runs in the library's sm_100a
kernels.
"""
from ._lib import (DTYPE_BF16, DTYPE_F16, DTYPE_F32, DTYPE_U8, FETCH_FILTERED, FETCH_GATHER,
                   FETCH_LOADS, FETCH_POINT, FORM_EXACT, FORM_FAST, FORM_PLAIN,
                   KERNEL_CONSISTENCY, KERNEL_INIT, KERNEL_INIT_COARSE, KERNEL_PACK,
                   KERNEL_PROPAGATE, L3dError, MAX_SOURCES, WEIGHT_F32, WEIGHT_Q8)
from .memory import memory_reserved, trim_memory
from .camera import Intrinsics, Pose, StereoView, look_at, relative_pose, scale_intrinsics
from .stereo import (STEREO_METHODS, DenseStereo, SolveOptions, StereoInput, StereoOptions,
                     StereoRun, StereoSettings)
from .tsdf import BRICK, BrickGrid, IntegrationView, TsdfVolume

__all__ = [
    "BRICK", "BrickGrid", "DenseStereo", "IntegrationView", "Intrinsics", "L3dError", "Pose",
    "STEREO_METHODS", "SolveOptions", "StereoInput", "StereoOptions", "StereoRun",
    "StereoSettings", "StereoView", "TsdfVolume", "look_at", "relative_pose", "scale_intrinsics",
    "DTYPE_U8", "DTYPE_F32", "DTYPE_F16", "DTYPE_BF16", "FORM_PLAIN", "FORM_FAST", "FORM_EXACT",
    "WEIGHT_F32",
    "WEIGHT_Q8", "FETCH_FILTERED", "FETCH_GATHER", "FETCH_POINT", "FETCH_LOADS", "KERNEL_INIT", "KERNEL_INIT_COARSE", "KERNEL_PROPAGATE", "KERNEL_PACK",
    "KERNEL_CONSISTENCY", "MAX_SOURCES", "memory_reserved", "trim_memory",
]
