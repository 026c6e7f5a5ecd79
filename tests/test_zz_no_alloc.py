"""The allocation-free entry point, maxi_diffusion_device_noalloc, against the
regular device entry point (run with -m gpu).

It exists for callers that cannot allocate device memory during their work;
its scratch is a fixed array inside the library, shared by all calls.  This
file is named so that pytest collects it last: if it fails, a run that stops
at the first failure has already run every other test.  It also passes when
run alone in a fresh process (the first call performs the per-device set-up).
"""
import ctypes

import numpy as np
import pytest
import torch

from maxibone_b200 import _lib, gauss_kernel
from maxibone_b200.synthetic import spheres_mask

pytestmark = pytest.mark.gpu

MAX_VOXELS = 1 << 23


def _regular(mask_t, kernel, reps):
    """The existing entry point, maxi_diffusion_device, with library-allocated workspace."""
    out = torch.empty(mask_t.shape, dtype=torch.uint16, device="cuda")
    field = torch.empty(mask_t.shape, dtype=torch.float32, device="cuda")
    nz, ny, nx = mask_t.shape
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().maxi_diffusion_device(mask_t.data_ptr(), 0, nz, ny, nx, kernel.ctypes.data,
                                                kernel.shape[0], reps, out.data_ptr(), field.data_ptr(),
                                                0, 0, None, 0, st))
    torch.cuda.synchronize()
    return out.cpu().numpy(), field.cpu().numpy()


def _noalloc(mask_t, kernel, reps, shape=None, fmt=0, out=None, field=None):
    """The allocation-free entry point; `mask_t` is a uint8 mask (fmt 0) or the
    bit-packed words of a volume of `shape` (fmt 1)."""
    shape = tuple(mask_t.shape) if shape is None else shape
    out = torch.empty(shape, dtype=torch.uint16, device="cuda") if out is None else out
    field = torch.empty(shape, dtype=torch.float32, device="cuda") if field is None else field
    nz, ny, nx = shape
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().maxi_diffusion_device_noalloc(mask_t.data_ptr(), fmt, nz, ny, nx, kernel.ctypes.data,
                                                        kernel.shape[0], reps, out.data_ptr(),
                                                        field.data_ptr(), st))
    torch.cuda.synchronize()
    return out.cpu().numpy(), field.cpu().numpy()


def _pack_padded(mask):
    """MSB-first uint32 words of the flat mask, zero-padded to whole words."""
    flat = (mask.reshape(-1) != 0).astype(np.uint64)
    flat = np.concatenate([flat, np.zeros((-flat.size) % 32, np.uint64)])
    w = (flat.reshape(-1, 32) << np.arange(31, -1, -1, dtype=np.uint64)).sum(axis=1)
    return torch.from_numpy(w.astype(np.uint32).view(np.int32)).cuda()


def test_noalloc_matches_regular_entry_point_on_two_calls_in_a_row():
    # Two different volumes back to back: the second call must not be affected
    # by what the first left in the shared scratch array.
    cases = [
        (spheres_mask((64, 72, 80), 12, (3, 9), seed=31), gauss_kernel(3.0).astype(np.float32), 4),
        (spheres_mask((40, 96, 130), 8, (2, 7), seed=32), gauss_kernel(2.0).astype(np.float32), 3),
    ]
    for mask, kernel, reps in cases:
        m = torch.from_numpy(mask).cuda()
        want_u16, want_field = _regular(m, kernel, reps)
        got_u16, got_field = _noalloc(m, kernel, reps)
        assert np.abs(got_field - want_field).max() <= 1e-5
        assert np.abs(got_u16.astype(np.int32) - want_u16.astype(np.int32)).max() <= 1
        assert np.all(got_u16[mask > 0] == 65535)


def test_noalloc_rejects_volumes_above_its_limit():
    k = gauss_kernel(1.0).astype(np.float32)
    dummy = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    nz, ny, nx = 129, 256, 256  # 8,454,144 voxels > 2^23
    assert nz * ny * nx > MAX_VOXELS
    rc = _lib.lib().maxi_diffusion_device_noalloc(dummy, 0, nz, ny, nx, k.ctypes.data, k.shape[0], 1,
                                                  dummy, None, None)
    assert rc == 1
    assert b"no-alloc limit" in _lib.lib().maxi_last_error()


def test_noalloc_bitpacked_mask_matches_regular_entry_point():
    # 23 x 37 x 45 = 38,295 voxels: not a whole number of 32-bit mask words.
    mask = spheres_mask((23, 37, 45), 6, (2, 6), seed=33)
    kernel = gauss_kernel(2.5).astype(np.float32)
    want_u16, want_field = _regular(torch.from_numpy(mask).cuda(), kernel, 3)
    for _ in range(2):
        got_u16, got_field = _noalloc(_pack_padded(mask), kernel, 3, shape=mask.shape, fmt=1)
        assert np.abs(got_field - want_field).max() <= 1e-5
        assert np.abs(got_u16.astype(np.int32) - want_u16.astype(np.int32)).max() <= 1
        assert np.all(got_u16[mask > 0] == 65535)


def test_noalloc_stays_inside_the_callers_buffers():
    from test_gpu_guard_bands import MASK_SENTINEL, Guarded, _bytes_equal

    shape = (24, 56, 72)
    mask = spheres_mask(shape, 8, (2, 7), seed=34)
    kernel = gauss_kernel(4.0).astype(np.float32)
    plain_u16, plain_field = _noalloc(torch.from_numpy(mask).cuda(), kernel, 2)
    gm = Guarded(shape, torch.uint8, MASK_SENTINEL, init=torch.from_numpy(mask).cuda())
    go = Guarded(shape, torch.uint16)
    gf = Guarded(shape, torch.float32)
    _noalloc(gm.t, kernel, 2, out=go.t, field=gf.t)
    assert go.intact() and gf.intact(), "write outside the output or the field output"
    assert _bytes_equal(go.t, torch.from_numpy(plain_u16).cuda())
    assert _bytes_equal(gf.t, torch.from_numpy(plain_field).cuda())


def test_noalloc_rejects_a_misaligned_bitpacked_mask():
    k = gauss_kernel(1.0).astype(np.float32)
    dummy = ctypes.c_void_p(258)  # never dereferenced: rejected before any GPU work
    rc = _lib.lib().maxi_diffusion_device_noalloc(dummy, 1, 4, 4, 32, k.ctypes.data, k.shape[0], 1,
                                                  ctypes.c_void_p(256), None, None)
    assert rc == 1
    assert b"aligned" in _lib.lib().maxi_last_error()
