"""tcgen05 tensor-core z/y passes for the 16-bit field forms (run with -m gpu).

The tensor-core passes compute each z/y pass as a banded Toeplitz product with
FP32 accumulation; they must agree with the CUDA-core passes of the same form
(both store the field in the same 16-bit type) and stay within the stated
error of the FP64 form.  Shapes cover partial x chunks (nx not a multiple of
128), axes shorter than and not multiple of the 128-output tile, and the
radius range the tensor-core path serves (1..128).
"""
import numpy as np
import pytest
import torch

from maxibone_b200 import _lib, device, gauss_kernel
from maxibone_b200.synthetic import random_mask, spheres_mask

pytestmark = pytest.mark.gpu

# Max abs error vs the FP64 form: the 2e-3 contract for BF16 with error-feedback
# rounding (the default); FP16 values are 8x finer.  Round-to-nearest storage
# (error_feedback=False, an opt-out outside the contract) drifts more.
VS_F64 = {"bf16": 2e-3, "f16": 5e-4}
VS_F64_NEAREST = {"bf16": 8e-3, "f16": 1e-3}
# Max abs difference between the tensor-core and CUDA-core forms (same storage
# type, each within its bound of FP64).
TC_VS_CC = {"bf16": 4e-3, "f16": 1e-3}
TC_X = _lib.PATH_TENSOR_CORES_X | _lib.PATH_FUSED_YX  # the x pass alone or fused with the y pass


def run(mask, kernel, reps, field, tensor_cores=True, error_feedback=True):
    """Runs one diffusion; with 16-bit fields asserts which passes ran (the
    tensor-core z and y passes and a tensor-core x pass, alone or fused with
    the y pass; or only CUDA-core passes), so that a silent fallback cannot make
    a tensor-core vs CUDA-core comparison compare a path with itself."""
    m = torch.from_numpy(np.ascontiguousarray(mask, np.uint8)).cuda()
    fo = torch.empty(mask.shape, dtype=torch.float64 if field == "f64" else torch.float32, device="cuda")
    out = torch.empty(mask.shape, dtype=torch.uint16, device="cuda")
    device.diffuse(m, kernel, reps, output=out, field=field, field_out=fo, tensor_cores=tensor_cores,
                   error_feedback=error_feedback)
    path = device.last_path()
    if field in ("bf16", "f16"):
        if tensor_cores:
            assert path & _lib.PATH_TENSOR_CORES_ZY and path & TC_X and not path & _lib.PATH_CUDA_CORES, hex(path)
        else:
            assert path & _lib.PATH_CUDA_CORES and not path & (_lib.PATH_TENSOR_CORES_ZY | TC_X), hex(path)
    torch.cuda.synchronize()
    device.tensor_core_status()
    return out.cpu().numpy(), fo.cpu().numpy()


@pytest.mark.parametrize("field", ["bf16", "f16"])
@pytest.mark.parametrize("shape,sigma", [((40, 70, 136), 1.0), ((130, 64, 128), 3.0), ((33, 129, 200), 8.0),
                                         ((8, 300, 64), 2.0), ((200, 24, 72), 8.0)])
@pytest.mark.parametrize("ef", [False, True])
def test_tensor_core_matches_cuda_core_and_fp64(field, shape, sigma, ef):
    mask = random_mask(shape, 0.02, seed=sum(shape))
    kernel = gauss_kernel(sigma).astype(np.float32)
    reps = 3
    _, want = run(mask, kernel, reps, "f64")
    tc_u16, tc = run(mask, kernel, reps, field, True, ef)
    _, cc = run(mask, kernel, reps, field, False, ef)
    ef = ef and kernel.shape[0] // 2 >= 4  # narrower kernels always round to nearest
    assert np.abs(tc - cc).max() <= (TC_VS_CC if ef else VS_F64_NEAREST)[field]
    assert np.abs(tc.astype(np.float64) - want).max() <= (VS_F64 if ef else VS_F64_NEAREST)[field]
    assert np.all(tc_u16[mask > 0] == 65535)
    assert np.all(tc[mask > 0] == 1.0)


@pytest.mark.parametrize("radius", [1, 5, 12, 16, 31, 32])
def test_tensor_core_radius_range(radius):
    mask = spheres_mask((64, 96, 128), 10, (3, 9), seed=radius)
    kernel = gauss_kernel(radius / 4.0).astype(np.float32)
    _, want = run(mask, kernel, 4, "f64")
    for field in ("f16", "bf16"):
        _, got = run(mask, kernel, 4, field, True, True)
        _, cc = run(mask, kernel, 4, field, False, True)
        # below radius 4 the stores round to nearest (error feedback needs the
        # next x pass to remove its noise, which a kernel that narrow does not)
        bound = VS_F64 if radius >= 4 else VS_F64_NEAREST
        assert np.abs(got - cc).max() <= (TC_VS_CC if radius >= 4 else VS_F64_NEAREST)[field]
        assert np.abs(got.astype(np.float64) - want).max() <= bound[field]


# Radii above 32: z / y passes with the Toeplitz halves in tensor memory (64-column
# tiles and two TMA boxes per K run above radius 64), the x pass in its transposed
# form with error feedback along the rows.
@pytest.mark.parametrize("radius", [33, 40, 64, 65, 96, 128])
@pytest.mark.parametrize("shape", [(48, 100, 264), (70, 131, 136)])
def test_tensor_core_wide_radius(radius, shape):
    mask = spheres_mask(shape, 10, (3, 12), seed=radius + shape[2])
    kernel = gauss_kernel(radius / 4.0).astype(np.float32)
    _, want = run(mask, kernel, 3, "f64")
    for field in ("f16", "bf16"):
        u16, got = run(mask, kernel, 3, field, True, True)
        _, cc = run(mask, kernel, 3, field, False, True)
        assert np.abs(got - cc).max() <= TC_VS_CC[field]
        assert np.abs(got.astype(np.float64) - want).max() <= VS_F64[field]
        assert np.all(u16[mask > 0] == 65535)


def test_tensor_core_wide_radius_repeats_bit_for_bit():
    mask = spheres_mask((64, 96, 200), 12, (3, 10), seed=11)
    kernel = gauss_kernel(32.0).astype(np.float32)
    a = run(mask, kernel, 4, "bf16")[1]
    b = run(mask, kernel, 4, "bf16")[1]
    np.testing.assert_array_equal(a, b)


def test_error_feedback_reduces_bf16_error():
    mask = spheres_mask((96, 96, 128), 30, (4, 14), seed=5)
    kernel = gauss_kernel(4.0).astype(np.float32)
    _, want = run(mask, kernel, 30, "f64")
    _, rn = run(mask, kernel, 30, "bf16", True, False)
    _, ef = run(mask, kernel, 30, "bf16", True, True)
    e_rn = np.abs(rn.astype(np.float64) - want).max()
    e_ef = np.abs(ef.astype(np.float64) - want).max()
    assert e_ef < e_rn


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_tensor_core_final_pass_outputs_optional(field):
    mask = random_mask((20, 40, 128), 0.03, seed=3)
    kernel = gauss_kernel(2.0).astype(np.float32)
    m = torch.from_numpy(mask).cuda()
    u16_only = torch.empty(mask.shape, dtype=torch.uint16, device="cuda")
    device.diffuse(m, kernel, 3, output=u16_only, field=field)
    fo_only = torch.empty(mask.shape, dtype=torch.float32, device="cuda")
    device.diffuse(m, kernel, 3, output=None, field_out=fo_only, field=field)
    both_u16, both_fo = run(mask, kernel, 3, field)
    np.testing.assert_array_equal(u16_only.cpu().numpy(), both_u16)
    np.testing.assert_array_equal(fo_only.cpu().numpy(), both_fo)


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_tensor_core_bitpacked_mask(field):
    mask = spheres_mask((24, 50, 136), 8, (3, 8), seed=6)
    kernel = gauss_kernel(3.0).astype(np.float32)
    m = torch.from_numpy(mask).cuda()
    packed = device.bitpack(m)
    out_p = torch.empty(mask.shape, dtype=torch.uint16, device="cuda")
    fo_p = torch.empty(mask.shape, dtype=torch.float32, device="cuda")
    device.diffuse(packed, kernel, 3, output=out_p, field_out=fo_p, field=field, shape=mask.shape)
    u, f = run(mask, kernel, 3, field)
    np.testing.assert_array_equal(out_p.cpu().numpy(), u)
    np.testing.assert_array_equal(fo_p.cpu().numpy(), f)
