"""The Gaussian + EDT field combination (src/processing_steps/0975_combine_fields.py:38-62)
on the GPU against its oracle and the reference-derived golden (run with -m gpu).
The combination is FP32 arithmetic in a fixed order followed by a truncating
conversion, so results must be bit-identical."""
import os
import warnings

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from maxibone_b200 import device, gauss_kernel
from maxibone_b200.fields import combine_fields, mask_cylinder
from maxibone_b200.synthetic import spheres_mask

pytestmark = pytest.mark.gpu


def test_combine_fields_matches_reference_golden():
    z = np.load(os.path.join(GOLDEN, "combine_fields_u16.npz"))
    np.testing.assert_array_equal(combine_fields(z["gauss"], z["edt"]), z["output"])


# nx % 8 == 0 takes 8-voxel vector steps; other widths the scalar path.  Non-square
# planes use generate_cylinder_mask(ny, nx).
@pytest.mark.parametrize("shape", [(16, 64, 64), (7, 33, 41), (5, 40, 56), (3, 96, 24), (2, 1, 16)])
def test_combine_fields_matches_oracle(shape):
    rng = np.random.default_rng(sum(shape))
    gauss = (rng.random(shape) ** 2 * 65535).astype(np.uint16)
    edt = (rng.random(shape) * 50000).astype(np.uint16)
    gauss.reshape(-1)[0] = 1  # never all zero
    edt.reshape(-1)[0] = 1
    with warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)  # a plane with nothing inside: 0 / 0 in numpy
        want = oracle.combine_fields(gauss, edt)
    np.testing.assert_array_equal(combine_fields(gauss, edt), want)


def test_combine_fields_on_a_diffusion_output():
    shape = (40, 96, 96)
    mask = spheres_mask(shape, 10, (3, 12), seed=21)
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    device.diffuse(torch.from_numpy(mask).cuda(), gauss_kernel(3.0).astype(np.float32), 6, output=out)
    gauss = out.cpu().numpy() * oracle.cylinder_mask(96)  # the pipeline saves result * cylinder_mask
    edt = (np.random.default_rng(4).random(shape) * 40000).astype(np.uint16) * oracle.cylinder_mask(96)
    edt = edt.astype(np.uint16)
    np.testing.assert_array_equal(combine_fields(gauss.astype(np.uint16), edt), oracle.combine_fields(
        gauss.astype(np.uint16), edt))


def test_combine_fields_device_tensors():
    rng = np.random.default_rng(9)
    gauss = rng.integers(1, 65535, (8, 48, 64), dtype=np.uint16)
    edt = rng.integers(1, 65535, (8, 48, 64), dtype=np.uint16)
    got = combine_fields(torch.from_numpy(gauss.view(np.int16)).cuda(), torch.from_numpy(edt.view(np.int16)).cuda())
    np.testing.assert_array_equal(got.cpu().numpy().view(np.uint16), oracle.combine_fields(gauss, edt))


def test_combine_fields_rejects_all_zero_field_and_bad_shapes():
    z = np.zeros((4, 16, 16), np.uint16)
    with pytest.raises(ValueError):
        combine_fields(z, z + 1)
    with pytest.raises(ValueError):
        combine_fields(z + 1, np.ones((4, 16, 8), np.uint16))
    with pytest.raises(TypeError):
        combine_fields(z.astype(np.float32), z)


# The diffusion step's result * generate_cylinder_mask(nx) (square planes, as the
# script) and the (ny, nx) form for other planes; odd and even sizes, one-voxel axes.
@pytest.mark.parametrize("shape", [(4, 64, 64), (3, 65, 65), (2, 40, 56), (2, 1, 16), (1, 7, 1), (5, 33, 100)])
def test_mask_cylinder_matches_reference_multiply(shape):
    rng = np.random.default_rng(sum(shape))
    field = rng.integers(0, 65536, shape, dtype=np.uint16)
    want = field * oracle.cylinder_mask(shape[1], shape[2])
    assert want.dtype == np.uint16
    np.testing.assert_array_equal(mask_cylinder(field), want)
    t = torch.from_numpy(field.view(np.int16)).cuda()
    assert mask_cylinder(t) is t
    np.testing.assert_array_equal(t.cpu().numpy().view(np.uint16), want)


def test_mask_cylinder_on_diffusion_output():
    shape = (32, 96, 96)
    mask = spheres_mask(shape, 10, (3, 12), seed=5)
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    device.diffuse(torch.from_numpy(mask).cuda(), gauss_kernel(2.0).astype(np.float32), 4, output=out)
    want = out.cpu().numpy() * oracle.cylinder_mask(96)
    mask_cylinder(out)
    np.testing.assert_array_equal(out.cpu().numpy(), want)
