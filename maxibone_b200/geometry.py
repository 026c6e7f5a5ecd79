"""The implant masks of the reference's geometry module on the GPU.

``compute_front_back_masks(mask, voxel_size, E, cm, cp, UVWp, front_mask,
back_mask, implant_shell_mask, solid_implant)`` keeps the pybind argument list of
src/pybind/geometry-pybind.cc:283-310 (computing src/lib/cpp/cpu_seq/geometry.cc:112-215)
and writes the four uint8 masks in place.  src/processing_steps/0750_bone_region.py:62
calls it to make the ``implant_solid`` mask that the diffusion step diffuses; the
results are identical to the reference's.

The mask is taken as uint8 (as the binding's forcecast); E, cm, cp and UVWp as
float32 (E and UVWp 3x3 row-major, cm and cp length 3, as the script passes them).
The outputs must be C-contiguous uint8 arrays of the mask's shape (numpy, or CUDA
tensors to stay on the device).  This module provides this one function of the
reference's geometry module; the others are not part of this library.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _f32(a, n, name):
    v = np.ascontiguousarray(np.asarray(a, dtype=np.float32).reshape(-1))
    if v.size != n:
        raise ValueError(f"{name} must have {n} values, got {v.size}")
    return v


def compute_front_back_masks(mask, voxel_size, E, cm, cp, UVWp, front_mask, back_mask, implant_shell_mask,
                             solid_implant) -> None:
    """Writes the front, back, implant-shell and solid-implant masks of `mask`."""
    import torch

    outs = (front_mask, back_mask, implant_shell_mask, solid_implant)
    on_device = isinstance(mask, torch.Tensor)
    if on_device:
        if not mask.is_cuda or mask.dtype != torch.uint8:
            raise TypeError("mask must be a uint8 CUDA tensor")
        m = mask.contiguous()
        for o in outs:
            if not isinstance(o, torch.Tensor) or not o.is_cuda or o.dtype != torch.uint8 or not o.is_contiguous():
                raise TypeError("outputs must be contiguous uint8 CUDA tensors with a CUDA mask")
        dev_outs = outs
    else:
        for o in outs:
            if not isinstance(o, np.ndarray) or o.dtype != np.uint8 or not o.flags.c_contiguous:
                raise TypeError("outputs must be C-contiguous uint8 numpy arrays")
        m = torch.from_numpy(np.ascontiguousarray(mask, dtype=np.uint8)).cuda()
        dev_outs = tuple(torch.empty_like(m) for _ in outs)
    if m.dim() != 3 or any(tuple(o.shape) != tuple(m.shape) for o in outs):
        raise ValueError(f"mask and outputs must be 3-D and of one shape, got {tuple(m.shape)}")
    e, c, p, u = _f32(E, 9, "E"), _f32(cm, 3, "cm"), _f32(cp, 3, "cp"), _f32(UVWp, 9, "UVWp")
    nz, ny, nx = m.shape
    ptr = lambda a: a.ctypes.data  # noqa: E731
    _lib.check(_lib.lib().maxi_implant_masks(m.data_ptr(), nz, ny, nx, float(np.float32(voxel_size)), ptr(e),
                                             ptr(c), ptr(p), ptr(u), *(o.data_ptr() for o in dev_outs),
                                             torch.cuda.current_stream().cuda_stream))
    if not on_device:
        for o, d in zip(outs, dev_outs):
            o[...] = d.cpu().numpy()
