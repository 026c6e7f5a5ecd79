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


def _noalloc(mask_t, kernel, reps):
    out = torch.empty(mask_t.shape, dtype=torch.uint16, device="cuda")
    field = torch.empty(mask_t.shape, dtype=torch.float32, device="cuda")
    nz, ny, nx = mask_t.shape
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().maxi_diffusion_device_noalloc(mask_t.data_ptr(), 0, nz, ny, nx, kernel.ctypes.data,
                                                        kernel.shape[0], reps, out.data_ptr(),
                                                        field.data_ptr(), st))
    torch.cuda.synchronize()
    return out.cpu().numpy(), field.cpu().numpy()


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
