"""The implant masks (src/lib/cpp/cpu_seq/geometry.cc:112-215 via
src/pybind/geometry-pybind.cc:283-310) on the GPU against the golden made by the
reference's own module and the oracle (run with -m gpu).  FP32 in the reference's
operation order: the masks must be identical."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from maxibone_b200.geometry import compute_front_back_masks

pytestmark = pytest.mark.gpu


def _frame(rng, implant):
    E = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    UVWp = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    cm = np.array(np.nonzero(implant)).mean(axis=1)
    return E, cm, rng.normal(size=3) * 5, UVWp


def _run(mask, vs, E, cm, cp, UVWp):
    outs = [np.full(mask.shape, 7, np.uint8) for _ in range(4)]
    compute_front_back_masks(mask, vs, E, cm, cp, UVWp, *outs)
    return outs


def test_implant_masks_match_reference_golden():
    z = np.load(os.path.join(GOLDEN, "implant_masks_u8.npz"))
    got = _run(z["mask"], float(z["voxel_size"]), z["E"], z["cm"], z["cp"], z["UVWp"])
    for g, name in zip(got, ("front", "back", "shell", "solid")):
        np.testing.assert_array_equal(g, z[name], err_msg=name)


# Tilted cylinders of several sizes, stray voxels and bytes other than 1, an empty
# mask (w0 = 0, rmax = 0), one-voxel axes.
@pytest.mark.parametrize("seed,shape", [(1, (24, 40, 48)), (2, (33, 31, 29)), (3, (16, 64, 64)), (4, (1, 30, 70)),
                                        (5, (40, 1, 33)), (6, (300, 20, 3))])
def test_implant_masks_match_oracle(seed, shape):
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    implant = ((((yy - ny / 2 - 0.1 * zz) ** 2 + (xx - nx / 2 + 1) ** 2) < (max(min(ny, nx), 4) / 4) ** 2)
               & (zz > 0)).astype(np.uint8)
    implant[rng.random(shape) > 0.995] = 1
    implant[rng.random(shape) > 0.998] = 3
    if not implant.any():
        implant.reshape(-1)[0] = 1
    E, cm, cp, UVWp = _frame(rng, implant)
    want = oracle.implant_masks(implant, 1.875, E, cm, cp, UVWp)
    for g, w in zip(_run(implant, 1.875, E, cm, cp, UVWp), want):
        np.testing.assert_array_equal(g, w)


def test_implant_masks_empty_mask_and_device_tensors():
    rng = np.random.default_rng(9)
    empty = np.zeros((6, 20, 24), np.uint8)
    E, _, cp, UVWp = _frame(rng, np.ones((2, 2, 2)))
    cm = np.array([3.0, 10.0, 12.0])
    want = oracle.implant_masks(empty, 2.5, E, cm, cp, UVWp)
    for g, w in zip(_run(empty, 2.5, E, cm, cp, UVWp), want):
        np.testing.assert_array_equal(g, w)
    m = np.zeros((10, 32, 32), np.uint8)
    m[2:8, 10:20, 12:22] = 1
    t = torch.from_numpy(m).cuda()
    outs = [torch.empty_like(t) for _ in range(4)]
    compute_front_back_masks(t, 1.0, E, cm, cp, UVWp, *outs)
    for g, w in zip(outs, oracle.implant_masks(m, 1.0, E, cm, cp, UVWp)):
        np.testing.assert_array_equal(g.cpu().numpy(), w)


def test_implant_masks_reject_bad_outputs():
    m = np.ones((2, 3, 4), np.uint8)
    eye = np.eye(3)
    with pytest.raises(TypeError):
        compute_front_back_masks(m, 1.0, eye, [1, 1, 1], [0, 0, 0], eye, *[np.zeros((2, 3, 4), bool)] * 4)
    with pytest.raises(ValueError):
        compute_front_back_masks(m, 1.0, eye, [1, 1, 1], [0, 0, 0], eye, *[np.zeros((2, 3, 5), np.uint8)] * 4)
    with pytest.raises(ValueError):
        compute_front_back_masks(m, 1.0, eye[:2], [1, 1, 1], [0, 0, 0], eye, *[np.zeros((2, 3, 4), np.uint8)] * 4)


def test_implant_masks_full_size_against_oracle_planes():
    """A 512 x 1024 x 1024 tilted implant: sampled planes equal the oracle's (which
    takes w0 from the whole mask and rmax from each plane)."""
    nz, ny, nx = 512, 1024, 1024
    z = torch.arange(nz, device="cuda", dtype=torch.float32)[:, None, None]
    y = torch.arange(ny, device="cuda", dtype=torch.float32)[None, :, None]
    x = torch.arange(nx, device="cuda", dtype=torch.float32)[None, None, :]
    t = ((((y - 512 - 0.15 * z) ** 2 + (x - 500) ** 2) < 120.0 ** 2) & (z > 20)).to(torch.uint8)
    rng = np.random.default_rng(12)
    E = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    UVWp = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    idx = torch.nonzero(t).to(torch.float64).mean(0).cpu().numpy()
    cp = rng.normal(size=3) * 20
    outs = [torch.empty_like(t) for _ in range(4)]
    compute_front_back_masks(t, 1.875, E, idx, cp, UVWp, *outs)
    planes = (0, 21, 255, 511)
    want = oracle.implant_masks(t.cpu().numpy(), 1.875, E, idx, cp, UVWp, planes=planes)
    for g, w in zip(outs, want):
        for i, zp in enumerate(planes):
            np.testing.assert_array_equal(g[zp].cpu().numpy(), w[i])
