"""Image preparation on the GPU, in front of the stereo stage (frontend/src/app/vision/image/
gray-image.ts rgbaToGray / downsampleRgb / downsampleGray, mvs/depth-maps.ts upsampleDepth), over
the l3d_image_* / l3d_depth_upsample entry points.  Inputs and outputs are CUDA tensors; the
kernels run on torch's current stream."""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib


def _stream() -> C.c_void_p:
    s = torch.cuda.current_stream().cuda_stream
    return C.c_void_p(s if s else 1)  # 1 = cudaStreamLegacy


def _cuda(t: torch.Tensor, dtype, name: str) -> torch.Tensor:
    if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CUDA {dtype} tensor")
    return t


def rgba_to_gray(rgba: torch.Tensor, width: int, height: int) -> torch.Tensor:
    """(H, W, 4) uint8 -> (height, width) uint8 luma, area-averaged."""
    _cuda(rgba, torch.uint8, "rgba")
    out = torch.empty((height, width), dtype=torch.uint8, device=rgba.device)
    _lib.check(_lib.load().l3d_image_rgba_to_gray(C.c_void_p(rgba.data_ptr()), rgba.shape[1],
                                                  rgba.shape[0], width, height,
                                                  C.c_void_p(out.data_ptr()), _stream()))
    return out


def downsample_rgb(rgba: torch.Tensor, width: int, height: int) -> torch.Tensor:
    """(H, W, 4) uint8 -> (height, width, 3) uint8 thumbnail."""
    _cuda(rgba, torch.uint8, "rgba")
    out = torch.empty((height, width, 3), dtype=torch.uint8, device=rgba.device)
    _lib.check(_lib.load().l3d_image_downsample_rgb(C.c_void_p(rgba.data_ptr()), rgba.shape[1],
                                                    rgba.shape[0], width, height,
                                                    C.c_void_p(out.data_ptr()), _stream()))
    return out


def downsample_gray(gray: torch.Tensor, width: int, height: int) -> torch.Tensor:
    _cuda(gray, torch.uint8, "gray")
    out = torch.empty((height, width), dtype=torch.uint8, device=gray.device)
    _lib.check(_lib.load().l3d_image_downsample_gray(C.c_void_p(gray.data_ptr()), gray.shape[1],
                                                     gray.shape[0], width, height,
                                                     C.c_void_p(out.data_ptr()), _stream()))
    return out


def upsample_depth(grid: torch.Tensor, width: int, height: int) -> torch.Tensor:
    """Phone depth grid (gh, gw) float32 metres (0 = none) -> (height, width) prior."""
    _cuda(grid, torch.float32, "grid")
    out = torch.empty((height, width), dtype=torch.float32, device=grid.device)
    _lib.check(_lib.load().l3d_depth_upsample(C.c_void_p(grid.data_ptr()), grid.shape[1], grid.shape[0],
                                              width, height, C.c_void_p(out.data_ptr()), _stream()))
    return out
