"""The sphere morphology (src/lib/cpp/cpu_seq/morphology.cc, gpu/morphology.cc via
src/pybind/morphology-pybind.cc) on the GPU against its oracle and the golden made by
the reference's own module (run with -m gpu).  Masks are bits: results must be identical."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from maxibone_b200 import _lib
from maxibone_b200 import morphology as mo
from maxibone_b200.synthetic import spheres_mask

pytestmark = pytest.mark.gpu


def _pack(bits):
    return np.packbits(bits.astype(np.uint8), axis=-1).view(">u4").astype(np.uint32).reshape(
        bits.shape[0], bits.shape[1], -1)


def _u8(fn, mask, r):
    out = np.zeros(mask.shape, np.uint8)
    fn(mask, r, out)
    return out


def test_morphology_matches_reference_golden():
    z = np.load(os.path.join(GOLDEN, "morphology_u8.npz"))
    for name in ("dilate_r3", "dilate_r16", "erode_r2", "erode_r5"):
        op, r = name.split("_r")
        fn = mo.dilate_3d_sphere if op == "dilate" else mo.erode_3d_sphere
        np.testing.assert_array_equal(_u8(fn, z["mask"], int(r)), z[name], err_msg=name)


# Rows that are not whole words, one-voxel axes, radii from 0 to the 32 maximum, bytes
# with bit 0 clear (nonzero for dilation, 0 for erosion).
@pytest.mark.parametrize("shape,r", [((9, 10, 11), 0), ((12, 14, 16), 1), ((20, 22, 24), 5), ((18, 20, 37), 16),
                                     ((8, 30, 70), 9), ((40, 1, 33), 3), ((1, 50, 64), 12), ((70, 70, 70), 32),
                                     ((33, 34, 100), 20)])
def test_morphology_matches_oracle(shape, r):
    rng = np.random.default_rng(r + shape[2])
    m = (rng.random(shape) > 0.6).astype(np.uint8)
    m[rng.random(shape) > 0.97] = 2
    m[rng.random(shape) > 0.99] = 255
    np.testing.assert_array_equal(_u8(mo.dilate_3d_sphere, m, r), oracle.morphology_sphere(m, r, True))
    dense = (rng.random(shape) > 0.05).astype(np.uint8)
    dense[rng.random(shape) > 0.98] = 2
    np.testing.assert_array_equal(_u8(mo.erode_3d_sphere, dense, r), oracle.morphology_sphere(dense, r, False))


@pytest.mark.parametrize("shape,r", [((10, 12, 64), 0), ((12, 14, 32), 1), ((20, 22, 96), 5), ((24, 30, 64), 15),
                                     ((24, 40, 128), 16), ((16, 20, 64), 20), ((40, 40, 64), 31), ((3, 5, 32), 2)])
def test_morphology_bitpacked_matches_oracle(shape, r):
    rng = np.random.default_rng(3 * r + shape[0])
    sparse = (rng.random(shape) > 0.97).astype(np.uint8)
    dense = (rng.random(shape) > 0.03).astype(np.uint8)
    for bits, dilate, fn in ((sparse, True, mo.dilate_3d_sphere_bitpacked),
                             (dense, False, mo.erode_3d_sphere_bitpacked)):
        words = _pack(bits)
        out = np.zeros_like(words)
        fn(words, r, out)
        np.testing.assert_array_equal(out, oracle.morphology_sphere_bitpacked(words, r, dilate))


def test_morphology_device_tensors_and_in_place():
    mask = spheres_mask((32, 48, 64), 6, (3, 8), seed=2)
    t = torch.from_numpy(mask).cuda()
    out = torch.empty_like(t)
    mo.dilate_3d_sphere(t, 4, out)
    want = oracle.morphology_sphere(mask, 4, True)
    np.testing.assert_array_equal(out.cpu().numpy(), want)
    words = torch.from_numpy(_pack(mask).view(np.int32)).cuda()
    mo.erode_3d_sphere_bitpacked(words, 3, words)  # in place: the input is read before the result is written
    np.testing.assert_array_equal(words.cpu().numpy().view(np.uint32),
                                  oracle.morphology_sphere_bitpacked(_pack(mask), 3, False))


def test_morphology_rejects_bad_arguments():
    m = np.ones((4, 4, 32), np.uint8)
    with pytest.raises(TypeError):  # the binding takes np_result without conversion
        mo.dilate_3d_sphere(m, 1, np.zeros((4, 4, 32), np.int16))
    with pytest.raises(ValueError):
        mo.dilate_3d_sphere(m, 1, np.zeros((4, 4, 31), np.uint8))
    with pytest.raises(_lib.MaxiError):
        mo.dilate_3d_sphere(m, 33, np.zeros_like(m))
    with pytest.raises(_lib.MaxiError):
        mo.erode_3d_sphere_bitpacked(np.ones((2, 2, 1), np.uint32), 32, np.zeros((2, 2, 1), np.uint32))


def test_morphology_full_size_properties():
    """512 x 1024 x 1024: dilation is the complement of the erosion of the complement
    (outside voxels take no part in either), the uint8 and bit-packed forms agree below
    radius 16, and a lone voxel dilates to the sphere's voxel count."""
    nz, ny, nx, r = 512, 1024, 1024, 16
    g = torch.Generator(device="cuda").manual_seed(3)
    m = (torch.rand((nz, ny, nx), generator=g, device="cuda") > 0.9995).to(torch.uint8)
    dil = torch.empty_like(m)
    mo.dilate_3d_sphere(m, r, dil)
    ero = torch.empty_like(m)
    mo.erode_3d_sphere(1 - m, r, ero)
    assert torch.equal(dil, 1 - ero)
    r2 = 15
    dil2 = torch.empty_like(m)
    mo.dilate_3d_sphere(m, r2, dil2)
    bits = torch.tensor([1 << (31 - b) for b in range(32)], device="cuda", dtype=torch.int64)

    def pack(u8):  # MSB-first words as int32 bit patterns
        w = (u8.view(nz, ny, nx // 32, 32).to(torch.int64) * bits).sum(-1)
        return (w - (w >= 2 ** 31).to(torch.int64) * 2 ** 32).to(torch.int32)

    words = pack(m)
    wout = torch.empty_like(words)
    mo.dilate_3d_sphere_bitpacked(words, r2, wout)
    assert torch.equal(wout, pack(dil2))
    one = torch.zeros((80, 80, 96), dtype=torch.uint8, device="cuda")
    one[40, 40, 48] = 1
    sph = torch.empty_like(one)
    mo.dilate_3d_sphere(one, r, sph)
    k = np.arange(-r, r + 1)
    assert int(sph.sum()) == int(((k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2) <= r * r).sum())
