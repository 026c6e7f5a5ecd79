"""Histograms of a voxel volume against the diffusion field, on the GPU.

``field_histogram(np_voxels, np_field, np_offset, np_bins, vrange, frange,
verbose)`` has the arguments, meaning and in-place accumulation of the
reference's pybind ``histograms.field_histogram`` (src/pybind/
histograms-pybind.cc:81-107, computing src/lib/cpp/cpu/histograms.cc:231-305),
which the pipeline calls per z-block as ``field_histogram_par_gpu(voxels, field,
(zstart, 0, 0), f_bins[i], (vmin, vmax), (fmin, fmax), verbose)``
(src/processing_steps/1000_compute_histograms.py:472). The counts are identical
to the reference's: every FP64 binning expression is evaluated with its own
arithmetic on the host for all 65536 uint16 values and each axis coordinate,
and the kernel gathers from those tables and counts with 64-bit atomics.

Arguments are numpy arrays (voxels and field uint16, bins uint64 of shape
[field_bins, voxel_bins], added to in place) or CUDA tensors (uint16/int16
voxels and field, uint64/int64 bins added to on the device).
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _device_u16(a, name):
    import torch

    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if a.dtype not in (torch.uint16, torch.int16):
            raise TypeError(f"{name} must be uint16 (or int16 holding uint16 bits)")
        return a.contiguous()
    arr = np.asarray(a)
    if arr.dtype != np.uint16:
        raise TypeError(f"{name} must be a uint16 array")
    return torch.from_numpy(np.ascontiguousarray(arr).view(np.int16)).cuda()


def field_histogram(np_voxels, np_field, np_offset, np_bins, vrange, frange, verbose: int = 0) -> None:
    """Adds the (field bin, voxel bin) counts of np_voxels against np_field to np_bins."""
    import torch

    v = _device_u16(np_voxels, "voxels")
    f = _device_u16(np_field, "field")
    if v.dim() != 3 or f.dim() != 3:
        raise ValueError(f"voxels and field must be 3-D, got {tuple(v.shape)} and {tuple(f.shape)}")
    _, y_start, x_start = (int(o) for o in np_offset)
    vmin, vmax = (float(x) for x in vrange)
    fmin, fmax = (float(x) for x in frange)
    on_device = isinstance(np_bins, torch.Tensor)
    if on_device:
        if not np_bins.is_cuda or np_bins.dtype not in (torch.uint64, torch.int64) or not np_bins.is_contiguous():
            raise TypeError("bins must be a contiguous uint64/int64 CUDA tensor")
        bins = np_bins
    else:
        if not isinstance(np_bins, np.ndarray) or np_bins.dtype != np.uint64 or not np_bins.flags.c_contiguous:
            raise TypeError("bins must be a C-contiguous uint64 numpy array")
        bins = torch.from_numpy(np_bins.view(np.int64)).cuda()
    if bins.dim() != 2:
        raise ValueError(f"bins must be 2-D [field_bins, voxel_bins], got {tuple(bins.shape)}")
    field_bins, voxel_bins = bins.shape
    nZ, nY, nX = v.shape
    nz, ny, nx = f.shape
    if verbose >= 2:
        print(f"field_histogram: voxels {tuple(v.shape)}, field {tuple(f.shape)}, bins {tuple(bins.shape)}, "
              f"vrange {(vmin, vmax)}, frange {(fmin, fmax)}")
    st = torch.cuda.current_stream()
    _lib.check(_lib.lib().maxi_field_histogram(v.data_ptr(), nZ, nY, nX, f.data_ptr(), nz, ny, nx, y_start, x_start,
                                               bins.data_ptr(), field_bins, voxel_bins, vmin, vmax, fmin, fmax,
                                               st.cuda_stream))
    if not on_device:
        np_bins.view(np.int64)[...] = bins.cpu().numpy()
