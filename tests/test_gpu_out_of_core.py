"""Out-of-core (z-slabs with deep halos) and on-disk forms (run with -m gpu).

The FP32 slab results must equal the in-memory results bit for bit: a core
voxel sees the same input planes in the same tap order.  The on-disk form is
checked against the oracle of the reference's on-disk semantics (mask rebuilt
as field == 1.0f each repetition, uint16 output)."""
import numpy as np
import pytest
import torch

import oracle
from maxibone_b200 import diffusion, gauss_kernel
from maxibone_b200.diffusion import diffusion_out_of_core
from maxibone_b200.synthetic import random_mask, spheres_mask

pytestmark = pytest.mark.gpu


# Planes of a multiple of 32 voxels take the shrinking plane windows; the others
# run every repetition over the whole slab.
@pytest.mark.parametrize("shape,slab,sigma,reps", [((70, 33, 48), 16, 1.5, 3), ((40, 20, 64), 7, 1.0, 5),
                                                    ((128, 64, 128), 40, 2.0, 2), ((9, 9, 9), 2, 1.0, 1),
                                                    ((200, 32, 64), 30, 2.0, 6), ((61, 16, 96), 5, 1.0, 9)])
def test_out_of_core_equals_in_memory_fp32(shape, slab, sigma, reps):
    mask = random_mask(shape, 0.05, seed=sum(shape))
    kernel = gauss_kernel(sigma).astype(np.float32)
    want = np.empty(shape, np.uint16)
    diffusion(mask, kernel, want, reps)
    got = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, got, (slab, shape[1], shape[2]), reps)
    np.testing.assert_array_equal(got, want)


def test_out_of_core_pinned_buffers_and_bf16():
    shape = (96, 40, 128)
    mask = spheres_mask(shape, 10, (3, 8), seed=2)
    kernel = gauss_kernel(2.0).astype(np.float32)
    pin_m = torch.empty(shape, dtype=torch.uint8, pin_memory=True)
    pin_m.copy_(torch.from_numpy(mask))
    pin_o = torch.zeros(shape, dtype=torch.int16, pin_memory=True)
    o = pin_o.numpy().view(np.uint16)
    diffusion_out_of_core(pin_m.numpy(), kernel, o, (20, 40, 128), 3, field="bf16")
    whole = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, whole, (96, 40, 128), 3, field="bf16")
    # Slabs change the z-pass tiling of the tensor-core path: results agree to a few LSB.
    assert np.abs(o.astype(np.int32) - whole.astype(np.int32)).max() <= 64
    assert np.all(o[mask > 0] == 65535)


@pytest.mark.parametrize("chunk", [3, 16])
def test_pinned_mask_uploaded_in_chunks_equals_in_memory_fp32(chunk, monkeypatch):
    # From a pinned mask the resident upload runs on its own stream, chunk by
    # chunk, and each slab waits only for the chunks it reads: small chunks
    # and thin slabs make the first slabs compute while later chunks upload.
    monkeypatch.setenv("MAXIBONE_OOC_UPLOAD_CHUNK_PLANES", str(chunk))
    shape = (150, 64, 96)
    mask = spheres_mask(shape, 12, (3, 9), seed=chunk)
    kernel = gauss_kernel(2.0).astype(np.float32)
    want = np.empty(shape, np.uint16)
    diffusion(mask, kernel, want, 4)
    pin_m = torch.empty(shape, dtype=torch.uint8, pin_memory=True)
    pin_m.copy_(torch.from_numpy(mask))
    pin_o = torch.zeros(shape, dtype=torch.int16, pin_memory=True)
    got = pin_o.numpy().view(np.uint16)
    diffusion_out_of_core(pin_m.numpy(), kernel, got, (25, 64, 96), 4)
    np.testing.assert_array_equal(got, want)


def test_on_disk_matches_reference_semantics(tmp_path):
    shape = (48, 30, 40)
    mask = spheres_mask(shape, 6, (2, 7), seed=3)
    kernel = gauss_kernel(1.5).astype(np.float32)
    fin, fout = tmp_path / "mask.uint8", tmp_path / "field.uint16"
    mask.tofile(fin)
    diffusion(str(fin), kernel, str(fout), shape, (10, shape[1], shape[2]), 4)
    got = np.fromfile(fout, dtype=np.uint16).reshape(shape)
    want = oracle.diffusion_on_disk_semantics(mask, kernel, 4)
    assert np.abs(got.astype(np.int32) - want.astype(np.int32)).max() <= 1


@pytest.mark.parametrize("field,sigma,reps", [("bf16", 2.0, 4), ("f16", 2.0, 4), ("bf16", 10.0, 2)])
def test_out_of_core_16bit_fields_match_in_memory_field(field, sigma, reps):
    # Shrinking windows (plane of 8192 voxels) on the tensor-core path; sigma 10
    # (radius 40) takes the wide-radius passes.
    shape = (160, 64, 128)
    mask = spheres_mask(shape, 14, (3, 9), seed=5)
    kernel = gauss_kernel(sigma).astype(np.float32)
    got = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, got, (24, 64, 128), reps, field=field)
    whole = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, whole, (160, 64, 128), reps, field=field)
    assert np.abs(got.astype(np.int32) - whole.astype(np.int32)).max() <= 64
    assert np.all(got[mask > 0] == 65535)


def test_on_disk_shrinking_windows_match_reference_semantics(tmp_path):
    shape = (64, 32, 48)
    mask = spheres_mask(shape, 8, (2, 7), seed=4)
    kernel = gauss_kernel(1.0).astype(np.float32)
    fin, fout = tmp_path / "mask.uint8", tmp_path / "field.uint16"
    mask.tofile(fin)
    diffusion(str(fin), kernel, str(fout), shape, (9, shape[1], shape[2]), 5)
    got = np.fromfile(fout, dtype=np.uint16).reshape(shape)
    want = oracle.diffusion_on_disk_semantics(mask, kernel, 5)
    assert np.abs(got.astype(np.int32) - want.astype(np.int32)).max() <= 1


def test_on_disk_short_file_is_an_io_error(tmp_path):
    from maxibone_b200._lib import MaxiError
    fin = tmp_path / "short.uint8"
    np.zeros(100, np.uint8).tofile(fin)
    with pytest.raises(MaxiError, match="IO"):
        diffusion(str(fin), gauss_kernel(1), str(tmp_path / "o"), (10, 10, 10), (5, 10, 10), 1)


def _plan(shape, kernel_size, reps, device_bytes, field="f32"):
    import ctypes
    from maxibone_b200 import _lib
    s, k, res = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    _lib.check(_lib.lib().maxi_out_of_core_plan(*shape, 0, kernel_size, reps, _lib.FIELD_TYPES[field], 0,
                                                device_bytes, ctypes.byref(s), ctypes.byref(k), ctypes.byref(res)))
    return s.value, k.value, bool(res.value)


@pytest.mark.parametrize("budget", [4_000_000, 2_500_000])
def test_exchange_rounds_equal_in_memory_fp32(budget, monkeypatch):
    # A device budget too small for R x radius halos makes the planner run the
    # repetitions in rounds of k < R, the field going through host memory
    # between rounds; FP32 results equal the in-memory form bit for bit.
    shape, reps = (96, 64, 64), 12
    kernel = gauss_kernel(1.0).astype(np.float32)  # radius 4
    S, k, _ = _plan(shape, kernel.shape[0], reps, budget)
    assert k < reps and S < shape[0], (S, k)
    mask = spheres_mask(shape, 12, (3, 9), seed=budget % 97)
    want = np.empty(shape, np.uint16)
    diffusion(mask, kernel, want, reps)
    monkeypatch.setenv("MAXIBONE_OOC_DEVICE_BUDGET", str(budget))
    got = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, got, (0, shape[1], shape[2]), reps)
    np.testing.assert_array_equal(got, want)


def test_exchange_rounds_bf16_within_bounds(monkeypatch):
    shape, reps = (80, 64, 128), 10
    kernel = gauss_kernel(1.5).astype(np.float32)  # radius 6
    mask = spheres_mask(shape, 10, (3, 9), seed=5)
    S, k, _ = _plan(shape, kernel.shape[0], reps, 4_000_000, field="bf16")
    assert k < reps
    want = np.empty(shape, np.uint16)
    diffusion(mask, kernel, want, reps)  # FP32 in memory
    monkeypatch.setenv("MAXIBONE_OOC_DEVICE_BUDGET", "4000000")
    got = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, got, (0, shape[1], shape[2]), reps, field="bf16")
    assert np.abs(got.astype(np.int32) - want.astype(np.int32)).max() <= 2e-3 * 65535
    assert np.all(got[mask > 0] == 65535)


def test_planner_auto_slab_pageable_and_pinned_agree():
    shape = (130, 32, 96)
    mask = random_mask(shape, 0.05, seed=6)
    kernel = gauss_kernel(2.0).astype(np.float32)
    want = np.empty(shape, np.uint16)
    diffusion(mask, kernel, want, 4)
    got = np.zeros(shape, np.uint16)
    diffusion_out_of_core(mask, kernel, got, (0, shape[1], shape[2]), 4)
    np.testing.assert_array_equal(got, want)


def test_on_disk_against_the_reference_cpu_on_disk_file(tmp_path):
    # The golden holds the uint8 file the reference CPU backend's on-disk overload
    # wrote (floor(v * 255)); this library's on-disk overload writes the GPU
    # backend's uint16 (floor(v * 65535)).  Since 65535 = 255 * 257,
    # floor(u16 / 257) is the same quantity, so the two agree to 1 unit wherever
    # the FP32 fields agree to summation order.
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "on_disk_cpu_u8.npz"))
    mask, kernel, reps, gz = z["mask"], z["kernel"], int(z["reps"]), int(z["global_z"])
    shape = mask.shape
    fin, fout = tmp_path / "mask.uint8", tmp_path / "field.uint16"
    mask.tofile(fin)
    diffusion(str(fin), kernel, str(fout), shape, (gz, shape[1], shape[2]), reps)
    got = np.fromfile(fout, dtype=np.uint16).reshape(shape)
    d = np.abs((got // 257).astype(np.int32) - z["output"].astype(np.int32))
    assert d.max() <= 1
    assert (d > 0).mean() < 1e-3
    assert np.all(got[mask > 0] == 65535)
