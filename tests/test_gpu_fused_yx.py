"""The fused y + x tensor-core kernel (16-bit fields, radius <= 32; run with -m gpu).

It computes the y and x convolutions of a z-plane tile in one kernel, the
intermediate field rounded to the storage type in tensor memory instead of in
HBM.  Its results must stay within the 16-bit forms' bounds of the FP64 form,
agree with the separate y and x passes (both round the intermediate field to
the same type, with error-feedback chains that start at different x), keep
mask voxels exact, and be deterministic.  Every run asserts that the fused
kernel is what ran (MAXI_PATH_FUSED_YX), so a fallback cannot pass unnoticed.
The fused kernel uses the single coefficient set (the default from radius 4);
the split high + low halves, which smaller radii always use, run the separate
passes.
"""
import numpy as np
import pytest
import torch

from maxibone_b200 import _lib, device, gauss_kernel
from maxibone_b200.synthetic import random_mask, spheres_mask

pytestmark = pytest.mark.gpu

VS_F64 = {"bf16": 2e-3, "f16": 5e-4}
FUSED_VS_SEPARATE = {"bf16": 4e-3, "f16": 1e-3}
FUSED = _lib.PATH_TENSOR_CORES_ZY | _lib.PATH_FUSED_YX
SINGLE_SET_MIN_RADIUS = 4


def run(mask, kernel, reps, field, fused=True, split=False, output=True, field_out=True, bitpacked=False):
    m = torch.from_numpy(np.ascontiguousarray(mask, np.uint8)).cuda()
    shape = tuple(mask.shape)
    fo = torch.empty(shape, dtype=torch.float64 if field == "f64" else torch.float32, device="cuda") \
        if field_out else None
    out = torch.empty(shape, dtype=torch.uint16, device="cuda") if output else None
    if bitpacked:
        m = device.bitpack(m)
    device.diffuse(m, kernel, reps, output=out, field=field, field_out=fo, fuse_passes=fused,
                   split_coefficients=split, shape=shape)
    path = device.last_path()
    if field in ("bf16", "f16"):
        if fused and not split and kernel.shape[0] // 2 >= SINGLE_SET_MIN_RADIUS:
            assert path & FUSED == FUSED and not path & _lib.PATH_TENSOR_CORES_X, hex(path)
        else:
            assert not path & _lib.PATH_FUSED_YX, hex(path)
    torch.cuda.synchronize()
    device.tensor_core_status()
    return (out.cpu().numpy() if output else None), (fo.cpu().numpy() if field_out else None)


@pytest.mark.parametrize("field", ["bf16", "f16"])
@pytest.mark.parametrize("shape,sigma", [((24, 128, 128), 8.0), ((17, 200, 264), 8.0), ((9, 130, 136), 3.0),
                                         ((40, 64, 72), 1.0), ((5, 300, 64), 6.0), ((12, 100, 392), 4.0)])
def test_fused_matches_fp64_and_separate_passes(field, shape, sigma):
    mask = spheres_mask(shape, 10, (3, 10), seed=sum(shape))
    mask[random_mask(shape, 0.005, seed=1) > 0] = 1
    kernel = gauss_kernel(sigma).astype(np.float32)
    reps = 4
    _, want = run(mask, kernel, reps, "f64")
    u16, got = run(mask, kernel, reps, field)
    _, sep = run(mask, kernel, reps, field, fused=False)
    assert np.abs(got.astype(np.float64) - want).max() <= VS_F64[field]
    assert np.abs(got - sep).max() <= FUSED_VS_SEPARATE[field]
    assert np.all(u16[mask > 0] == 65535)
    assert np.all(got[mask > 0] == 1.0)


@pytest.mark.parametrize("radius", [1, 2, 4, 7, 8, 12, 16, 20, 24, 31, 32])
def test_fused_radius_range(radius):
    shape = (20, 150, 200)
    mask = spheres_mask(shape, 10, (3, 9), seed=radius)
    kernel = gauss_kernel(radius / 4.0).astype(np.float32)
    assert kernel.shape[0] == 2 * radius + 1
    _, want = run(mask, kernel, 3, "f64")
    # below radius 4 the 16-bit stores round to nearest (no error feedback)
    bound = VS_F64 if radius >= 4 else {"bf16": 8e-3, "f16": 1e-3}
    for field in ("bf16", "f16"):
        u16, got = run(mask, kernel, 3, field)
        assert np.abs(got.astype(np.float64) - want).max() <= bound[field], field
        assert np.all(u16[mask > 0] == 65535)


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_single_and_split_coefficients_within_bounds(field):
    # The default single 16-bit coefficient set (sum and second moment kept,
    # fused y + x kernel) and the split high + low halves (separate passes)
    # both stay within the bound of the FP64 form, and close to each other.
    from maxibone_b200.synthetic import bone_implant_mask
    mask = bone_implant_mask((128, 128, 256), seed=4, implant_radius=20.0).numpy()
    kernel = gauss_kernel(8.0).astype(np.float32)
    _, want = run(mask, kernel, 40, "f64")
    u16, got = run(mask, kernel, 40, field)
    u16s, split = run(mask, kernel, 40, field, split=True)
    assert np.abs(got.astype(np.float64) - want).max() <= VS_F64[field]
    assert np.abs(split.astype(np.float64) - want).max() <= VS_F64[field]
    assert np.all(u16[mask > 0] == 65535) and np.all(u16s[mask > 0] == 65535)


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_fused_outputs_optional_and_bitpacked_mask(field):
    mask = spheres_mask((14, 96, 136), 8, (3, 8), seed=7)
    kernel = gauss_kernel(3.0).astype(np.float32)
    both_u16, both_fo = run(mask, kernel, 3, field)
    u16_only, _ = run(mask, kernel, 3, field, field_out=False)
    _, fo_only = run(mask, kernel, 3, field, output=False)
    np.testing.assert_array_equal(u16_only, both_u16)
    np.testing.assert_array_equal(fo_only, both_fo)
    bp_u16, bp_fo = run(mask, kernel, 3, field, bitpacked=True)
    np.testing.assert_array_equal(bp_u16, both_u16)
    np.testing.assert_array_equal(bp_fo, both_fo)


def test_fused_repeats_bit_for_bit():
    mask = spheres_mask((30, 260, 264), 20, (3, 12), seed=9)
    kernel = gauss_kernel(8.0).astype(np.float32)
    a = run(mask, kernel, 5, "bf16")
    b = run(mask, kernel, 5, "bf16")
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_fused_one_repetition_and_empty_full_masks():
    kernel = gauss_kernel(2.0).astype(np.float32)
    for fill in (0, 1):
        mask = np.full((6, 64, 128), fill, np.uint8)
        u16, fo = run(mask, kernel, 2, "bf16")
        assert np.all(u16 == (65535 if fill else 0))
    mask = random_mask((8, 70, 128), 0.02, seed=2)
    _, want = run(mask, kernel, 1, "f64")
    _, got = run(mask, kernel, 1, "bf16")
    assert np.abs(got.astype(np.float64) - want).max() <= VS_F64["bf16"]


@pytest.mark.parametrize("field", ["bf16", "f16"])
@pytest.mark.parametrize("shape,sigma", [((1, 1, 64), 3.0), ((3, 33, 64), 8.0), ((2, 257, 1000), 4.0),
                                         ((4, 129, 136), 5.0)])
def test_fused_thin_and_ragged_shapes(field, shape, sigma):
    # One plane, one row, the narrowest x extent the tensor-core passes take,
    # and extents one past a tile: windows and stores clipped on every side.
    mask = spheres_mask(shape, 4, (1, 4), seed=sum(shape)) if min(shape) > 2 else \
        random_mask(shape, 0.1, seed=sum(shape))
    kernel = gauss_kernel(sigma).astype(np.float32)
    _, want = run(mask, kernel, 3, "f64")
    u16, got = run(mask, kernel, 3, field)
    _, sep = run(mask, kernel, 3, field, fused=False)
    assert np.abs(got.astype(np.float64) - want).max() <= VS_F64[field]
    assert np.abs(got - sep).max() <= FUSED_VS_SEPARATE[field]
    assert np.all(u16[mask > 0] == 65535)
