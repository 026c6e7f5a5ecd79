"""Parity of the CUDA library against the oracle (run with -m gpu on a B200).

Criteria (from the reference's test, src/test/test_diffusion.py:90-98, and
the path's FP32 contract):
  * FP32 field: max |GPU - oracle| <= 1e-5 (summation order and FMA only);
  * uint16 output: within 1 LSB of the oracle;
  * mask voxels: exactly 65535 (re-illumination is bit-exact);
  * reference-rounding mode: bit-identical to the oracle (and so to the
    reference module) in both the field and the uint16 output;
  * FP64 form: within 1e-12 of the CPU FP64 oracle;
  * BF16 / FP16 field forms: max abs error vs FP64 within the stated bounds.
"""
import numpy as np
import pytest
import torch

import oracle
from conftest import DIFFUSION_CASES, load_golden
from maxibone_b200 import _lib, device, diffusion, gauss_kernel
from maxibone_b200.synthetic import random_mask, spheres_mask

pytestmark = pytest.mark.gpu

F32_TOL = 1e-5
# Max abs error vs the FP64 form, per storage type (field values lie in [0, 1]):
# the BF16 contract is 2e-3; FP16's stored values are 8x finer.
LOWP_TOL = {"bf16": 2e-3, "f16": 5e-4}


def run_gpu(mask, kernel, reps, field="f32", mask_format="u8", reference_rounding=False, tensor_cores=True):
    m = torch.from_numpy(np.ascontiguousarray(mask, np.uint8)).cuda()
    shape = tuple(mask.shape)
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    fo = torch.empty(shape, dtype=torch.float64 if field == "f64" else torch.float32, device="cuda")
    if mask_format == "bitpacked":
        m = device.bitpack(m)
    device.diffuse(m, kernel, reps, output=out, field=field, field_out=fo, shape=shape,
                   reference_rounding=reference_rounding, tensor_cores=tensor_cores)
    torch.cuda.synchronize()
    return out.cpu().numpy(), fo.cpu().numpy()


def assert_parity(mask, kernel, reps, got_u16, got_field, want_u16, want_field):
    np.testing.assert_array_less(np.abs(got_field.astype(np.float64) - want_field), F32_TOL + 1e-30)
    assert np.abs(got_u16.astype(np.int32) - want_u16.astype(np.int32)).max(initial=0) <= 1
    if reps > 0:
        assert np.all(got_u16[np.asarray(mask) > 0] == 65535)


@pytest.mark.parametrize("name", DIFFUSION_CASES)
def test_golden_cases_fp32(name):
    mask, kernel, reps, golden, entry = load_golden(name)
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, reps)
    got_u16, got_field = run_gpu(mask, kernel, reps)
    assert_parity(mask, kernel, reps, got_u16, got_field, want_u16, want_field)
    if golden is not None:
        assert np.abs(got_u16.astype(np.int32) - golden.astype(np.int32)).max(initial=0) <= 1


@pytest.mark.parametrize("name", DIFFUSION_CASES)
def test_golden_cases_reference_rounding_bit_exact(name):
    mask, kernel, reps, golden, entry = load_golden(name)
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, reps)
    got_u16, got_field = run_gpu(mask, kernel, reps, reference_rounding=True)
    np.testing.assert_array_equal(got_u16, want_u16)
    np.testing.assert_array_equal(got_field, want_field)
    if golden is not None:
        np.testing.assert_array_equal(got_u16, golden)


# Every unrolled radius bucket, radii between buckets (zero-padded taps), and
# radii above the unrolled set (generic pass).
@pytest.mark.parametrize("radius", [1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 16, 20, 24, 32, 40, 48, 64, 96, 128, 140])
def test_radius_coverage(radius):
    shape = (19, 37, 300) if radius > 40 else (23, 45, 77)
    mask = random_mask(shape, 0.03, seed=radius)
    kernel = gauss_kernel(radius / 4.0).astype(np.float32)
    assert kernel.shape[0] == 2 * radius + 1
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, 2)
    got_u16, got_field = run_gpu(mask, kernel, 2)
    assert_parity(mask, kernel, 2, got_u16, got_field, want_u16, want_field)


# z / y axes spanning several 256-output tiles with a partial last tile (520,
# 530, 1030, 600) and x extents that leave a partial 32-column tile.
@pytest.mark.parametrize("shape,sigma", [((520, 530, 40), 8.0), ((1030, 8, 24), 3.0), ((6, 600, 36), 1.0)])
def test_long_axes(shape, sigma):
    mask = spheres_mask(shape, 120, (3, 12), seed=sum(shape))
    kernel = gauss_kernel(sigma).astype(np.float32)
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, 2)
    got_u16, got_field = run_gpu(mask, kernel, 2)
    assert_parity(mask, kernel, 2, got_u16, got_field, want_u16, want_field)


@pytest.mark.parametrize("shape", [(1, 1, 1), (1, 1, 40), (1, 40, 1), (40, 1, 1), (2, 3, 5), (33, 17, 70),
                                   (130, 7, 9), (5, 129, 260), (3, 2, 513)])
def test_edge_shapes(shape):
    mask = random_mask(shape, 0.1, seed=sum(shape))
    kernel = gauss_kernel(3).astype(np.float32)  # radius 12: larger than several axes
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, 3)
    got_u16, got_field = run_gpu(mask, kernel, 3)
    assert_parity(mask, kernel, 3, got_u16, got_field, want_u16, want_field)


@pytest.mark.parametrize("fill", [0, 1])
def test_empty_and_full_masks(fill):
    mask = np.full((20, 21, 22), fill, np.uint8)
    kernel = gauss_kernel(2).astype(np.float32)
    got_u16, got_field = run_gpu(mask, kernel, 4)
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, 4)
    assert_parity(mask, kernel, 4, got_u16, got_field, want_u16, want_field)
    if fill == 0:
        assert not got_u16.any()
    else:
        assert np.all(got_u16 == 65535)


def test_non_binary_mask_values_count_as_set():
    mask = random_mask((16, 16, 16), 0.2, seed=3) * np.uint8(7)
    mask[0, 0, :8] = 255
    kernel = gauss_kernel(1.5).astype(np.float32)
    want_u16, want_field = oracle.diffusion_in_memory(mask, kernel, 3)
    got_u16, got_field = run_gpu(mask, kernel, 3)
    assert_parity(mask, kernel, 3, got_u16, got_field, want_u16, want_field)


def test_bitpacked_mask_equals_u8_mask():
    mask = spheres_mask((40, 44, 50), 10, (3, 8), seed=4)  # 88000 voxels: words straddle rows
    kernel = gauss_kernel(2).astype(np.float32)
    a_u16, a_field = run_gpu(mask, kernel, 5)
    b_u16, b_field = run_gpu(mask, kernel, 5, mask_format="bitpacked")
    np.testing.assert_array_equal(a_u16, b_u16)
    np.testing.assert_array_equal(a_field, b_field)


def test_device_bitpack_matches_reference_layout():
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "bitpack_u32.npz"))
    packed = device.bitpack(torch.from_numpy(z["mask"]).cuda())
    np.testing.assert_array_equal(packed.cpu().numpy().view(np.uint32), z["packed"])
    decoded = device.bitunpack(torch.from_numpy(z["packed"].view(np.int32)).cuda(), z["mask"].size)
    np.testing.assert_array_equal(decoded.cpu().numpy(), z["decoded"])


def test_dropin_bitpacking_module_matches_reference_golden():
    # The pybind-style module through the reference's import path.
    import importlib
    import os
    from conftest import GOLDEN

    from maxibone_b200 import reference_imports
    reference_imports.install()
    bitpacking = importlib.import_module("lib.cpp.gpu.bitpacking")
    z = np.load(os.path.join(GOLDEN, "bitpack_u32.npz"))
    packed = np.zeros(z["packed"].shape, np.uint32)
    bitpacking.encode(z["mask"], packed)
    np.testing.assert_array_equal(packed, z["packed"])
    decoded = np.full(z["mask"].shape, 7, np.uint8)
    bitpacking.decode(z["packed"], decoded)
    np.testing.assert_array_equal(decoded, z["decoded"])


def test_fp64_form_matches_cpu_fp64_oracle():
    mask = spheres_mask((24, 28, 36), 8, (2, 6), seed=8)
    k64 = gauss_kernel(2.0)
    want = oracle.diffusion_f64(mask, k64.astype(np.float32).astype(np.float64), 6)
    _, got = run_gpu(mask, k64.astype(np.float32), 6, field="f64")
    assert np.abs(got - want).max() < 1e-12


def tensor_cores_ran(path: int) -> bool:
    """z and y passes on the tensor cores and the x pass too, alone or fused
    with the y pass."""
    return bool(path & _lib.PATH_TENSOR_CORES_ZY) and bool(path & (_lib.PATH_TENSOR_CORES_X | _lib.PATH_FUSED_YX))


@pytest.mark.parametrize("field", ["bf16", "f16"])
@pytest.mark.parametrize("shape,tc", [((48, 48, 48), False), ((48, 64, 128), True)])
def test_low_precision_fields_vs_fp64(field, shape, tc):
    mask = spheres_mask(shape, 12, (3, 8), seed=9)
    kernel = gauss_kernel(2.0).astype(np.float32)
    _, want = run_gpu(mask, kernel, 20, field="f64")
    got_u16, got = run_gpu(mask, kernel, 20, field=field, tensor_cores=tc)
    path = device.last_path()
    if tc:
        assert tensor_cores_ran(path), hex(path)
    else:
        assert path & _lib.PATH_CUDA_CORES and not tensor_cores_ran(path) and not path & _lib.PATH_FP32_FALLBACK, \
            hex(path)
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= LOWP_TOL[field], err.max()
    assert np.all(got_u16[mask > 0] == 65535)
    assert np.all(got[mask > 0] == 1.0)


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_low_precision_contract_case(field):
    # The case where the error bound binds: a 256^3 bone-implant mask, sigma 8
    # (65 taps), R = 100 -- the contract's kernel and repetition count on a
    # smaller volume -- on the tensor-core passes, against the FP64 form.
    from maxibone_b200.synthetic import bone_implant_mask
    mask = bone_implant_mask((256, 256, 256), seed=3, implant_radius=30.0).numpy()
    kernel = gauss_kernel(8.0).astype(np.float32)
    _, want = run_gpu(mask, kernel, 100, field="f64")
    got_u16, got = run_gpu(mask, kernel, 100, field=field)
    assert tensor_cores_ran(device.last_path())
    device.tensor_core_status()
    err = np.abs(got.astype(np.float64) - want)
    assert err.max() <= LOWP_TOL[field], err.max()
    assert np.all(got_u16[mask > 0] == 65535)


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_low_precision_request_on_a_shape_without_tensor_cores_runs_fp32(field):
    # nx = 40 is below the tensor-core passes' 64-column minimum: the request is
    # served by the FP32 form, which is faster and more accurate than the
    # 16-bit CUDA-core passes, and says so through the path bits.
    mask = spheres_mask((30, 50, 40), 8, (3, 8), seed=10)
    kernel = gauss_kernel(3.0).astype(np.float32)
    u16, got = run_gpu(mask, kernel, 5, field=field)
    assert device.last_path() & _lib.PATH_FP32_FALLBACK
    u16_f32, want = run_gpu(mask, kernel, 5, field="f32")
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(u16, u16_f32)


def test_dropin_host_call_matches_oracle():
    mask, kernel, reps, golden, entry = load_golden("spheres_32x40x48_s2_r5")
    out = np.zeros(mask.shape, np.uint16)
    diffusion(mask.astype(bool), kernel.astype(np.float64), out, reps)
    assert np.abs(out.astype(np.int32) - golden.astype(np.int32)).max() <= 1


def test_dropin_pageable_buffers_staged_equal_pinned():
    # Above 64 MB the drop-in call moves pageable numpy buffers through pinned
    # staging with several host threads; pinned buffers are copied directly.
    # Both routes give the same bits, here with an odd byte count so that the
    # last staging chunk is partial.
    shape = (257, 512, 512)
    mask = random_mask(shape, 0.02, seed=7)
    kernel = gauss_kernel(2.0).astype(np.float32)
    pageable_out = np.empty(shape, np.uint16)  # pages not yet touched, as np.empty leaves them
    diffusion(mask, kernel, pageable_out, 1)
    pin_m = torch.empty(shape, dtype=torch.uint8, pin_memory=True)
    pin_m.copy_(torch.from_numpy(mask))
    pin_o = torch.zeros(shape, dtype=torch.int16, pin_memory=True)
    diffusion(pin_m.numpy(), kernel, pin_o.numpy().view(np.uint16), 1)
    np.testing.assert_array_equal(pageable_out, pin_o.numpy().view(np.uint16))
    assert np.all(pageable_out[mask > 0] == 65535)


def test_dropin_zero_repetitions():
    mask = random_mask((5, 6, 7), 0.5, seed=1)
    out = np.zeros(mask.shape, np.uint16)
    diffusion(mask, gauss_kernel(1), out, 0)
    np.testing.assert_array_equal(out, mask.astype(np.uint16) * 65535)


def test_workspace_reuse_and_stream():
    mask = random_mask((30, 31, 32), 0.05, seed=12)
    kernel = gauss_kernel(2).astype(np.float32)
    m = torch.from_numpy(mask).cuda()
    ws = torch.empty(device.workspace_bytes(mask.shape, "f32"), dtype=torch.uint8, device="cuda")
    s = torch.cuda.Stream()
    outs = []
    for _ in range(2):
        out = torch.empty(mask.shape, dtype=torch.uint16, device="cuda")
        with torch.cuda.stream(s):
            device.diffuse(m, kernel, 3, output=out, workspace=ws)
        s.synchronize()
        outs.append(out.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    want, _ = oracle.diffusion_in_memory(mask, kernel, 3)
    assert np.abs(outs[0].astype(np.int32) - want.astype(np.int32)).max() <= 1
    with pytest.raises(ValueError):
        device.diffuse(m, kernel, 3, output=out, workspace=ws[:100])


@pytest.mark.parametrize("field", ["f32", "f64"])
def test_field_out_without_uint16_output(field):
    mask = random_mask((12, 20, 300), 0.05, seed=21)
    kernel = gauss_kernel(2).astype(np.float32)
    m = torch.from_numpy(mask).cuda()
    fo = torch.empty(mask.shape, dtype=torch.float64 if field == "f64" else torch.float32, device="cuda")
    device.diffuse(m, kernel, 3, output=None, field=field, field_out=fo)
    _, want = oracle.diffusion_in_memory(mask, kernel, 3)
    assert np.abs(fo.cpu().numpy() - want).max() < 1e-5


@pytest.mark.parametrize("keep", [0, 1])
def test_dropin_repeated_calls_reuse_and_grow_cached_buffers(keep):
    # keep 0 (the default): buffers are allocated and freed per call, as the
    # reference does; keep 1: one grow-only allocation reused across calls.
    k = gauss_kernel(2).astype(np.float32)
    assert _lib.lib().maxi_keep_device_buffers(keep) == 0
    free0 = torch.cuda.mem_get_info()[0]
    for shape in [(20, 30, 40), (10, 10, 10), (40, 50, 60), (20, 30, 40)]:
        mask = random_mask(shape, 0.05, seed=sum(shape))
        out = np.zeros(shape, np.uint16)
        diffusion(mask, k, out, 3)
        want, _ = oracle.diffusion_in_memory(mask, k, 3)
        assert np.abs(out.astype(np.int32) - want.astype(np.int32)).max() <= 1
    if not keep:
        # nothing stays allocated on the device after the calls (allow the
        # allocator's granularity of slack)
        assert torch.cuda.mem_get_info()[0] >= free0 - (4 << 20)
    assert _lib.lib().maxi_release_cached_memory() == 0
    out = np.zeros((8, 8, 8), np.uint16)
    diffusion(random_mask((8, 8, 8), 0.2, seed=1), k, out, 2)  # allocates again after the release
    assert _lib.lib().maxi_keep_device_buffers(0) == 0
