"""The reference's histograms module on the GPU: the field histogram of a voxel
volume against the diffusion field, and the per-axis / radial histograms.

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

``axis_histograms(np_voxels, np_offset, np_x_bins, np_y_bins, np_z_bins,
np_r_bins, center, vrange, verbose)`` is the pybind ``histograms.axis_histograms``
(src/pybind/histograms-pybind.cc:30-66, computing src/lib/cpp/cpu/
histograms.cc:14-80), called per z-block as ``axis_histogram_par_gpu(voxels,
(zstart, 0, 0), x_bins, y_bins, z_bins, r_bins, center, (vmin, vmax), verbose)``
(src/processing_steps/1000_compute_histograms.py:470): the global shape is
(len(z_bins), len(y_bins), len(x_bins)), the voxel block covers planes zstart
onward with the global y and x extents, and the radial bin of (y, x) is
floor(sqrt((x - cx)^2 + (y - cy)^2)) for center = (cy, cx).

Arguments are numpy arrays (voxels and field uint16, bins uint64, added to in
place) or CUDA tensors (uint16/int16 voxels and field, uint64/int64 bins added
to on the device).
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


def _bins(b, name):
    """(device tensor, numpy array to copy back into or None) for one bins argument."""
    import torch

    if isinstance(b, torch.Tensor):
        if not b.is_cuda or b.dtype not in (torch.uint64, torch.int64) or not b.is_contiguous():
            raise TypeError(f"{name} must be a contiguous uint64/int64 CUDA tensor")
        t, host = b, None
    else:
        if not isinstance(b, np.ndarray) or b.dtype != np.uint64 or not b.flags.c_contiguous:
            raise TypeError(f"{name} must be a C-contiguous uint64 numpy array")
        t, host = torch.from_numpy(b.view(np.int64)).cuda(), b
    if t.dim() != 2:
        raise ValueError(f"{name} must be 2-D, got {tuple(t.shape)}")
    return t, host


def _copy_back(t, host):
    if host is not None:
        host.view(np.int64)[...] = t.cpu().numpy()


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
    bins, host = _bins(np_bins, "bins")
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
    _copy_back(bins, host)


def axis_histograms(np_voxels, np_offset, np_x_bins, np_y_bins, np_z_bins, np_r_bins, center, vrange,
                    verbose: int = 0) -> None:
    """Adds the x, y, z and radial histograms of the voxel block to the four bins arrays."""
    import torch

    v = _device_u16(np_voxels, "voxels")
    pairs = [_bins(b, n) for b, n in ((np_x_bins, "x_bins"), (np_y_bins, "y_bins"), (np_z_bins, "z_bins"),
                                      (np_r_bins, "r_bins"))]
    (xb, _), (yb, _), (zb, _), (rb, _) = pairs
    voxel_bins = xb.shape[1]
    if any(t.shape[1] != voxel_bins for t, _ in pairs):
        raise ValueError("all four bins arrays need the same number of voxel bins")
    Nz, Ny, Nx, n_r = zb.shape[0], yb.shape[0], xb.shape[0], rb.shape[0]
    if v.dim() != 3 or tuple(v.shape[1:]) != (Ny, Nx):
        raise ValueError(f"voxels must be [nz, {Ny}, {Nx}] (len(y_bins), len(x_bins)), got {tuple(v.shape)}")
    z_start, y_start, x_start = (int(o) for o in np_offset)
    cy, cx = (int(c) for c in center)
    if cy < 0 or cx < 0:
        raise TypeError("center is unsigned")
    vmin, vmax = (float(x) for x in vrange)
    if verbose >= 2:
        print(f"axis_histograms: block {tuple(v.shape)} at z {z_start}, global {(Nz, Ny, Nx)}, Nr {n_r}, "
              f"center {(cy, cx)}, vrange {(vmin, vmax)}")
    st = torch.cuda.current_stream()
    _lib.check(_lib.lib().maxi_axis_histograms(v.data_ptr(), v.shape[0], Nz, Ny, Nx, z_start, y_start, x_start,
                                               xb.data_ptr(), yb.data_ptr(), zb.data_ptr(), rb.data_ptr(),
                                               voxel_bins, n_r, cy, cx, vmin, vmax, st.cuda_stream))
    for t, host in pairs:
        _copy_back(t, host)
