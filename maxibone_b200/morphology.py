"""The reference's morphology module on the GPU: 3-D sphere dilation and erosion of
uint8 and bit-packed masks.

The four functions keep the pybind names and argument lists of
src/pybind/morphology-pybind.cc:147-150 -- ``dilate_3d_sphere(np_voxels, radius,
np_result)``, ``erode_3d_sphere``, ``dilate_3d_sphere_bitpacked`` and
``erode_3d_sphere_bitpacked`` -- and write into np_result in place (a C-contiguous
uint8 / uint32 array of the input's shape, taken without conversion, as the
binding's ``noconvert``).  The pipeline reaches them through
src/lib/py/helpers.py:19,205-229,326-375 (``import lib.cpp.gpu.morphology``,
``morph_3d``), served here by ``maxibone_b200.reference_imports.install()``.

uint8 masks: result = 1 where some in-volume voxel of the sphere of `radius` is
nonzero (dilation) / every one has bit 0 set (erosion), else 0.  Bit-packed masks
(uint32 words, MSB first along x): the GPU build's semantics, whose per-row kernel
holds x offsets -radius .. 31 - radius.  Numpy arrays go through the device and
back; CUDA tensors stay on the device.  Radii up to 32 (31 bit-packed) per call.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _run(np_voxels, radius, np_result, dilate: bool, packed: bool) -> None:
    import torch

    np_dtype, t_dtypes = (np.uint32, (torch.uint32, torch.int32)) if packed else (np.uint8, (torch.uint8,))
    name = "uint32" if packed else "uint8"
    r = int(radius)
    if isinstance(np_result, torch.Tensor):
        if not np_result.is_cuda or np_result.dtype not in t_dtypes or not np_result.is_contiguous():
            raise TypeError(f"np_result must be a contiguous {name} CUDA tensor")
        src = np_voxels if isinstance(np_voxels, torch.Tensor) else torch.from_numpy(
            np.ascontiguousarray(np_voxels, dtype=np_dtype).view(np.int32 if packed else np.uint8)).cuda()
        if src.dtype not in t_dtypes or not src.is_cuda:
            raise TypeError(f"np_voxels must be a {name} CUDA tensor")
        src, out, host = src.contiguous(), np_result, None
    else:
        if not isinstance(np_result, np.ndarray) or np_result.dtype != np_dtype or not np_result.flags.c_contiguous:
            raise TypeError(f"np_result must be a C-contiguous {name} numpy array")
        vox = np.ascontiguousarray(np_voxels, dtype=np_dtype)  # the binding's forcecast of the input
        view = np.int32 if packed else np.uint8
        src = torch.from_numpy(vox.view(view)).cuda()
        out, host = torch.empty_like(src), np_result
    if src.dim() != 3 or tuple(src.shape) != tuple(out.shape):
        raise ValueError(f"voxels and result must be 3-D and of one shape, got {tuple(src.shape)} and "
                         f"{tuple(out.shape)}")
    nz, ny, nx = src.shape
    fn = _lib.lib().maxi_morphology_sphere_bitpacked if packed else _lib.lib().maxi_morphology_sphere
    _lib.check(fn(src.data_ptr(), out.data_ptr(), nz, ny, nx, r, 1 if dilate else 0,
                  torch.cuda.current_stream().cuda_stream))
    if host is not None:
        host.view(np.int32 if packed else np.uint8)[...] = out.cpu().numpy()


def dilate_3d_sphere(np_voxels, radius, np_result) -> None:
    """Sphere dilation of a uint8 mask into np_result (uint8 0/1)."""
    _run(np_voxels, radius, np_result, True, False)


def erode_3d_sphere(np_voxels, radius, np_result) -> None:
    """Sphere erosion of a uint8 mask into np_result (uint8 0/1)."""
    _run(np_voxels, radius, np_result, False, False)


def dilate_3d_sphere_bitpacked(np_voxels, radius, np_result) -> None:
    """Sphere dilation of a bit-packed uint32 mask into np_result."""
    _run(np_voxels, radius, np_result, True, True)


def erode_3d_sphere_bitpacked(np_voxels, radius, np_result) -> None:
    """Sphere erosion of a bit-packed uint32 mask into np_result."""
    _run(np_voxels, radius, np_result, False, True)
