"""Drop-in replacement for the reference's pybind module ``bitpacking``.

Mirrors src/pybind/bitpacking-pybind.cc:49-61 (the uint32 overloads that the
module registers): ``encode(np_mask, np_packed, verbose=0)`` and
``decode(np_packed, np_mask, verbose=0)``.  Both arguments are taken without
conversion, as pybind's ``.noconvert()``: np_mask must be a C-contiguous uint8
array and np_packed a C-contiguous uint32 array, else TypeError.  The packed
layout is the reference's: 32 voxels per word over the flat voxel order, MSB
first, and encode keeps bit 0 of each mask byte (``mask & 1``,
src/lib/cpp/cpu_seq/bitpacking.cc:9-42).

Unlike the reference, sizes are checked (its asserts vanish in release
builds): np_packed must hold at least np_mask.size bits and np_mask.size must
be a multiple of 32, else ValueError.  The work runs on the GPU through
``libmaxibone_diffusion.so`` (the arrays are copied to the device and back);
there is no CPU fallback.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def _check(np_mask, np_packed):
    if not isinstance(np_mask, np.ndarray) or np_mask.dtype != np.uint8 or not np_mask.flags.c_contiguous:
        raise TypeError("np_mask must be a C-contiguous numpy.ndarray of dtype uint8 (it is not converted)")
    if not isinstance(np_packed, np.ndarray) or np_packed.dtype != np.uint32 or not np_packed.flags.c_contiguous:
        raise TypeError("np_packed must be a C-contiguous numpy.ndarray of dtype uint32 (it is not converted)")
    if np_mask.size % 32 != 0:
        raise ValueError(f"np_mask has {np_mask.size} elements, not a multiple of 32")
    if np_packed.size * 32 < np_mask.size:
        raise ValueError(f"np_packed holds {np_packed.size * 32} bits, fewer than the {np_mask.size} mask voxels")


def encode(np_mask, np_packed, verbose=0):
    """Packs bit 0 of each byte of np_mask into np_packed (in place), MSB first."""
    import torch

    _check(np_mask, np_packed)
    n = np_mask.size
    if n == 0:
        return
    d_mask = torch.from_numpy(np_mask.reshape(-1)).cuda()
    d_packed = torch.empty(n // 32, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    _lib.check(_lib.lib().maxi_bitpack_encode(d_mask.data_ptr(), n, d_packed.data_ptr(), st.cuda_stream))
    np_packed.reshape(-1)[: n // 32] = d_packed.cpu().numpy().view(np.uint32)
    if verbose:
        print(f"bitpacking.encode: {n} voxels -> {n // 32} words")


def decode(np_packed, np_mask, verbose=0):
    """Unpacks np_packed into np_mask (in place): one uint8 {0, 1} per voxel."""
    import torch

    _check(np_mask, np_packed)
    n = np_mask.size
    if n == 0:
        return
    d_packed = torch.from_numpy(np_packed.reshape(-1)[: n // 32].view(np.int32)).cuda()
    d_mask = torch.empty(n, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream()
    _lib.check(_lib.lib().maxi_bitpack_decode(d_packed.data_ptr(), n, d_mask.data_ptr(), st.cuda_stream))
    np_mask.reshape(-1)[:] = d_mask.cpu().numpy()
    if verbose:
        print(f"bitpacking.decode: {n // 32} words -> {n} voxels")
