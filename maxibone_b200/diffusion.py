"""Drop-in replacement for the reference's pybind module ``diffusion``.

Mirrors src/pybind/diffusion-pybind.cc:81-85: one function ``diffusion`` with
two overloads, the same argument names (including ``repititions``), defaults
and conversion rules:

* ``diffusion(np_voxels, np_kernel, np_output, repititions=1, verbose=0)``
  In-memory form (diffusion-pybind.cc:27-53).  ``np_voxels`` and ``np_kernel``
  are force-cast to C-contiguous uint8 / float32 (so bool masks and float64
  kernels are accepted, as pybind's ``forcecast`` does); ``np_output`` is not
  converted: it must already be a C-contiguous uint16 array, else TypeError
  (pybind's ``.noconvert()``).  The output is written in place.
* ``diffusion(input_file, np_kernel, output_file, total_shape, global_shape,
  repititions=1, verbose=0)``  On-disk form (diffusion-pybind.cc:67-77): reads
  a raw uint8 file, writes a raw uint16 file.

Unlike the reference, malformed arguments raise ValueError instead of being
undefined behaviour (shape mismatch, non-3-D volumes, even-length kernels).
The work runs on the GPU through ``libmaxibone_diffusion.so``; there is no CPU
fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib


def _as_int(v, name):
    if isinstance(v, (bool, np.bool_)) or not isinstance(v, (int, np.integer)):
        raise TypeError(f"diffusion(): incompatible function arguments: {name} must be an int")
    return int(v)


def _in_memory(np_voxels, np_kernel, np_output, repititions=1, verbose=0):
    if not isinstance(np_output, np.ndarray) or np_output.dtype != np.uint16 or not np_output.flags.c_contiguous:
        raise TypeError("diffusion(): incompatible function arguments: np_output must be a C-contiguous "
                        "numpy.ndarray of dtype uint16 (it is not converted)")
    if not np_output.flags.writeable:
        raise ValueError("np_output is read-only")
    voxels = np.ascontiguousarray(np_voxels, dtype=np.uint8)
    kernel = np.ascontiguousarray(np_kernel, dtype=np.float32)
    reps = _as_int(repititions, "repititions")
    verbose = _as_int(verbose, "verbose")
    if voxels.ndim != 3:
        raise ValueError(f"np_voxels must be 3-D (z, y, x), got shape {voxels.shape}")
    if kernel.ndim != 1:
        raise ValueError(f"np_kernel must be 1-D, got shape {kernel.shape}")
    if np_output.shape != voxels.shape:
        raise ValueError(f"np_output shape {np_output.shape} differs from np_voxels shape {voxels.shape}")
    nz, ny, nx = voxels.shape
    lib = _lib.lib()
    _lib.check(lib.maxi_diffusion_in_memory(
        voxels.ctypes.data, nz, ny, nx, kernel.ctypes.data, kernel.shape[0], reps,
        np_output.ctypes.data, verbose))


def _on_disk(input_file, np_kernel, output_file, total_shape, global_shape, repititions=1, verbose=0):
    kernel = np.ascontiguousarray(np_kernel, dtype=np.float32)
    if kernel.ndim != 1:
        raise ValueError(f"np_kernel must be 1-D, got shape {kernel.shape}")
    ts = tuple(_as_int(v, "total_shape") for v in total_shape)
    gs = tuple(_as_int(v, "global_shape") for v in global_shape)
    if len(ts) != 3 or len(gs) != 3:
        raise ValueError("total_shape and global_shape must be (z, y, x) tuples")
    lib = _lib.lib()
    _lib.check(lib.maxi_diffusion_on_disk(
        os.fsencode(input_file), kernel.ctypes.data, kernel.shape[0], os.fsencode(output_file),
        ts[0], ts[1], ts[2], gs[0], gs[1], gs[2],
        _as_int(repititions, "repititions"), _as_int(verbose, "verbose")))


def diffusion_out_of_core(np_voxels, np_kernel, np_output, global_shape, repititions=1, verbose=0, field="f32"):
    """Out-of-core form for host volumes larger than the device (the reference's
    NS::diffusion_out_of_core, src/lib/cpp/include/diffusion.hh:74): z-slabs of
    global_shape[0] planes with deep halos, streamed through the GPU."""
    if not isinstance(np_output, np.ndarray) or np_output.dtype != np.uint16 or not np_output.flags.c_contiguous:
        raise TypeError("np_output must be a C-contiguous numpy.ndarray of dtype uint16")
    voxels = np.ascontiguousarray(np_voxels, dtype=np.uint8)
    kernel = np.ascontiguousarray(np_kernel, dtype=np.float32)
    if voxels.ndim != 3 or np_output.shape != voxels.shape:
        raise ValueError("np_voxels must be 3-D and np_output of the same shape")
    gz = _as_int(global_shape[0], "global_shape")
    nz, ny, nx = voxels.shape
    _lib.check(_lib.lib().maxi_diffusion_out_of_core_ex(
        voxels.ctypes.data, nz, ny, nx, gz, kernel.ctypes.data, kernel.shape[0], _as_int(repititions, "repititions"),
        np_output.ctypes.data, _lib.FIELD_TYPES[field], 0, _as_int(verbose, "verbose")))


def diffusion(*args, **kwargs):
    """Repeated separable 3-D Gaussian with re-illumination, quantised to uint16.

    Overloads (as the reference pybind module):
      diffusion(np_voxels, np_kernel, np_output, repititions=1, verbose=0) -> None
      diffusion(input_file, np_kernel, output_file, total_shape, global_shape,
                repititions=1, verbose=0) -> None
    """
    first = args[0] if args else kwargs.get("np_voxels", kwargs.get("input_file"))
    if isinstance(first, (str, bytes, os.PathLike)):
        return _on_disk(*args, **kwargs)
    return _in_memory(*args, **kwargs)
