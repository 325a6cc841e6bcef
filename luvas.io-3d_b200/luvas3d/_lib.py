"""ctypes binding of libluvas3d.so (the C ABI declared in include/luvas3d.h).

The library is loaded from luvas3d/lib/ next to this file.  There is no fallback: if the
shared library is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(_HERE, "lib")
LIB_PATH = os.path.join(LIB_DIR, "libluvas3d.so")

L3D_OK, L3D_EINVAL, L3D_ECUDA, L3D_ENOMEM, L3D_ESTATE, L3D_ETIMEOUT = range(6)
DTYPE_U8, DTYPE_F32, DTYPE_F16, DTYPE_BF16 = range(4)
FORM_PLAIN, FORM_FAST, FORM_EXACT = 0, 1, 2
WEIGHT_F32, WEIGHT_Q8 = 0, 1
KERNEL_INIT, KERNEL_INIT_COARSE, KERNEL_PROPAGATE, KERNEL_PACK, KERNEL_CONSISTENCY = range(5)
MAX_SOURCES = 8
FETCH_FILTERED, FETCH_GATHER, FETCH_POINT, FETCH_LOADS = range(4)
NOALLOC_MAX_BRICKS = 1 << 20


class L3dError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[status {status}] {message}")
        self.status = status


class Intrinsics(C.Structure):
    _fields_ = [("fx", C.c_double), ("fy", C.c_double), ("cx", C.c_double), ("cy", C.c_double)]


class Pose(C.Structure):
    _fields_ = [("R", C.c_double * 9), ("t", C.c_double * 3)]


class View(C.Structure):
    _fields_ = [("intrinsics", Intrinsics), ("pose", Pose)]


class StereoOpts(C.Structure):
    _fields_ = [
        ("coarse", C.c_void_p),
        ("depth_maps", C.c_int32),
        ("storage", C.c_int32),
        ("form", C.c_int32),
        ("window", C.c_int32),
        ("dilation", C.c_int32),
        ("stream", C.c_void_p),
        ("compensated", C.c_int32),
    ]


class SolveOpts(C.Structure):
    _fields_ = [
        ("sources", C.POINTER(C.c_int32)),
        ("n_sources", C.c_int32),
        ("min_depth", C.c_double),
        ("max_depth", C.c_double),
        ("prior", C.POINTER(C.c_float)),
        ("geometric", C.c_int32),
        ("iterations", C.c_int32),
        ("from_coarse", C.c_int32),
        ("pack", C.c_int32),
    ]


class StereoBuffers(C.Structure):
    _fields_ = [
        ("images", C.c_void_p),
        ("depths", C.c_void_p),
        ("hyp", C.c_void_p),
        ("cost", C.c_void_p),
        ("filtered", C.c_void_p),
        ("filtered_all", C.c_void_p),
        ("hyp_all", C.c_void_p),
        ("cost_all", C.c_void_p),
    ]


class TsdfDesc(C.Structure):
    _fields_ = [
        ("origin", C.c_double * 3),
        ("voxel", C.c_double),
        ("truncation", C.c_double),
        ("max_weight", C.c_double),
        ("prior_weight", C.c_double),
        ("dense", C.c_int32),
        ("dims", C.c_int32 * 3),
        ("coords", C.POINTER(C.c_int32)),
        ("count", C.c_int32),
        ("weight_type", C.c_int32),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("stream", C.c_void_p),
    ]


class SdfBricks(C.Structure):
    _fields_ = [
        ("origin", C.c_double * 3),
        ("voxel", C.c_double),
        ("dims", C.c_int32 * 3),
        ("lookup", C.c_void_p),
        ("tsdf", C.c_void_p),
        ("weight", C.c_void_p),
        ("bricks", C.c_int64),
    ]


class IntegrationView(C.Structure):
    _fields_ = [
        ("intrinsics", Intrinsics),
        ("pose", Pose),
        ("max_depth", C.c_double),
        ("prior", C.POINTER(C.c_float)),
        ("confidence", C.c_double),
    ]


# (name, restype, argtypes); every symbol here is declared in include/luvas3d.h
_P = C.c_void_p
_I = C.c_int32
SIGNATURES = [
    ("l3d_last_error", C.c_size_t, [C.c_char_p, C.c_size_t]),
    ("l3d_stereo_opts_default", None, [C.POINTER(StereoOpts)]),
    ("l3d_stereo_create", C.c_int, [_I, _I, _I, C.POINTER(View), C.POINTER(StereoOpts), C.POINTER(_P)]),
    ("l3d_stereo_create_sized", C.c_int, [_I, C.POINTER(View), C.POINTER(C.c_int32),
                                          C.POINTER(StereoOpts), C.POINTER(_P)]),
    ("l3d_stereo_view_size", C.c_int, [_P, _I, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("l3d_stereo_set_image", C.c_int, [_P, _I, _I, _P, C.c_int64]),
    ("l3d_stereo_solve", C.c_int, [_P, _I, C.POINTER(SolveOpts)]),
    ("l3d_stereo_solve_all", C.c_int, [_P, _I, C.POINTER(C.c_int32), C.POINTER(SolveOpts)]),
    ("l3d_stereo_dispatch", C.c_int, [_P, _I, _I, C.POINTER(SolveOpts), _I, _I]),
    ("l3d_stereo_filter", C.c_int, [_P, _I, C.POINTER(C.c_int32), _I, _I]),
    ("l3d_stereo_filter_all", C.c_int, [_P, _I, C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("l3d_stereo_read_filtered", C.c_int, [_P, _P]),
    ("l3d_stereo_read_filtered_layer", C.c_int, [_P, _I, _P]),
    ("l3d_stereo_read_filtered_all_async", C.c_int, [_P, _P]),
    ("l3d_stereo_read_depth", C.c_int, [_P, _I, _P]),
    ("l3d_stereo_read_hyp", C.c_int, [_P, _P, _P]),
    ("l3d_stereo_read_hyp_layer", C.c_int, [_P, _I, _P, _P]),
    ("l3d_stereo_write_hyp", C.c_int, [_P, _P, _P]),
    ("l3d_stereo_write_depth", C.c_int, [_P, _I, _P]),
    ("l3d_stereo_plane_cost", C.c_int, [_P, _I, C.POINTER(SolveOpts), _P, _P, _P]),
    ("l3d_stereo_buffers_get", C.c_int, [_P, C.POINTER(StereoBuffers)]),
    ("l3d_stereo_stream", C.c_int, [_P, C.POINTER(_P)]),
    ("l3d_stereo_synchronize", C.c_int, [_P]),
    ("l3d_stereo_launches", C.c_int64, [_P]),
    ("l3d_stereo_set_variant", C.c_int, [_P, _I]),
    ("l3d_stereo_variant", C.c_int32, [_P]),
    ("l3d_stereo_autotune", C.c_int, [_P, _I, C.POINTER(C.c_int32), C.POINTER(SolveOpts),
                                      C.POINTER(C.c_int32), C.POINTER(C.c_float)]),
    ("l3d_stereo_set_graphs", C.c_int, [_P, _I]),
    ("l3d_stereo_destroy", None, [_P]),
    ("l3d_tsdf_create", C.c_int, [C.POINTER(TsdfDesc), C.POINTER(_P)]),
    ("l3d_tsdf_integrate", C.c_int, [_P, _P, _P, C.POINTER(IntegrationView)]),
    ("l3d_tsdf_integrate_many", C.c_int, [_P, _P, C.POINTER(C.c_int32), _P, _I, C.POINTER(IntegrationView)]),
    ("l3d_tsdf_integrate_layer", C.c_int, [_P, _P, _I, C.POINTER(IntegrationView)]),
    ("l3d_tsdf_count_updates", C.c_int, [_P, _P, C.POINTER(C.c_int32), _P, _I, C.POINTER(IntegrationView),
                                         C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("l3d_tsdf_integrate_many_read", C.c_int, [_P, _P, C.POINTER(C.c_int32), _P, _I, C.POINTER(IntegrationView), _P, _P]),
    ("l3d_tsdf_integrate_many_read_async", C.c_int, [_P, _P, C.POINTER(C.c_int32), _P, _I, C.POINTER(IntegrationView), _P, _P]),
    ("l3d_tsdf_wait_read", C.c_int, [_P]),
    ("l3d_tsdf_read", C.c_int, [_P, _P, _P]),
    ("l3d_tsdf_reset", C.c_int, [_P]),
    ("l3d_tsdf_voxels", C.c_int64, [_P]),
    ("l3d_tsdf_device_buffers", C.c_int, [_P, C.POINTER(_P), C.POINTER(_P)]),
    ("l3d_tsdf_stream", C.c_int, [_P, C.POINTER(_P)]),
    ("l3d_tsdf_synchronize", C.c_int, [_P]),
    ("l3d_tsdf_launches", C.c_int64, [_P]),
    ("l3d_tsdf_destroy", None, [_P]),
    ("l3d_tsdf_integrate_noalloc", C.c_int, [C.POINTER(TsdfDesc), _P, _P, _P,
                                             C.POINTER(IntegrationView), _P, _P, _P]),
    ("l3d_cloud_create", C.c_int, [C.c_double, _P, C.POINTER(_P)]),
    ("l3d_cloud_add", C.c_int, [_P, _P, _P, _I, _I, C.POINTER(View), _P, _I, _I]),
    ("l3d_cloud_add_points", C.c_int, [_P, C.c_int64, _P]),
    ("l3d_cloud_coarsen", C.c_int, [_P, C.c_double]),
    ("l3d_cloud_size", C.c_int, [_P, C.POINTER(C.c_int64)]),
    ("l3d_cloud_cell", C.c_int, [_P, C.POINTER(C.c_double)]),
    ("l3d_cloud_read", C.c_int, [_P, _I, C.c_int64, C.POINTER(C.c_int64), _P, _P, _P, _P, _P]),
    ("l3d_cloud_launches", C.c_int64, [_P]),
    ("l3d_cloud_destroy", None, [_P]),
    ("l3d_extract_surface", C.c_int, [C.POINTER(SdfBricks), C.c_double, C.POINTER(_P)]),
    ("l3d_tsdf_extract_surface", C.c_int, [_P, C.c_double, C.POINTER(_P)]),
    ("l3d_mesh_counts", C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("l3d_mesh_read", C.c_int, [_P, _P, _P, _P]),
    ("l3d_mesh_remove_small_components", C.c_int, [_P, C.c_double, _I, C.POINTER(_P)]),
    ("l3d_mesh_launches", C.c_int64, [_P]),
    ("l3d_mesh_destroy", None, [_P]),
    ("l3d_brick_grid_build", C.c_int, [_P, C.c_double, _P, _P, C.c_int64, C.c_double, _P, _P, _P, _P]),
    ("l3d_image_rgba_to_gray", C.c_int, [_P, _I, _I, _I, _I, _P, _P]),
    ("l3d_image_downsample_rgb", C.c_int, [_P, _I, _I, _I, _I, _P, _P]),
    ("l3d_image_downsample_gray", C.c_int, [_P, _I, _I, _I, _I, _P, _P]),
    ("l3d_depth_upsample", C.c_int, [_P, _I, _I, _I, _I, _P, _P]),
    ("l3d_measure_texture_rate", C.c_int, [_I, _I, C.POINTER(C.c_double)]),
    ("l3d_measure_fetch_rate", C.c_int, [_I, _I, _I, C.POINTER(C.c_double)]),
    ("l3d_memory_trim", C.c_int, [C.c_int64]),
    ("l3d_memory_reserved", C.c_int, [C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    ("l3d_ncc_forward", C.c_int, [_P, _I, C.POINTER(C.c_int32), _I, _P, _P, _P, _P]),
    ("l3d_ncc_backward", C.c_int, [_P, _I, C.POINTER(C.c_int32), _I, _P, _P, _P, _P, _P, _P, _P]),
    ("l3d_tsdf_forward_depth", C.c_int, [_P, C.POINTER(IntegrationView), _I, _I, _P, _P, _P, _P, _P,
                                         _P, _P, _P]),
    ("l3d_tsdf_backward", C.c_int, [_P, C.POINTER(IntegrationView), _I, _I, _P, _P, _P, _P, _P, _P,
                                    _P, _P, _P, _P, _P]),
]

_lib = None


def load() -> C.CDLL:
    """Loads libluvas3d.so once; raises if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python luvas.io-3d_b200/build.py` "
                "(the CUDA kernels are the only implementation)")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().l3d_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(status: int) -> None:
    if status != L3D_OK:
        raise L3dError(status, last_error())


def ptr(array) -> C.c_void_p:
    """Address of a C-contiguous numpy array (or None)."""
    if array is None:
        return None
    if not array.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return C.c_void_p(array.ctypes.data)
