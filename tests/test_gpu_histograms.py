"""The field histogram (src/lib/cpp/cpu/histograms.cc:231-305 via
src/pybind/histograms-pybind.cc:81-107) on the GPU against its oracle and the
golden made by the reference's own module (run with -m gpu).  Counts are
integers from the reference's FP64 bin expressions, so they must be identical."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from maxibone_b200.histograms import field_histogram

pytestmark = pytest.mark.gpu


def _run(voxels, field, offset, bins_shape, vrange, frange, start=None):
    bins = np.zeros(bins_shape, np.uint64) if start is None else start.copy()
    field_histogram(voxels, field, offset, bins, vrange, frange, 0)
    return bins


def test_field_histogram_matches_reference_golden():
    z = np.load(os.path.join(GOLDEN, "field_histogram_u64.npz"))
    got = _run(z["voxels"], z["field"], (0, 0, 0), z["bins"].shape, tuple(z["vrange"]), tuple(z["frange"]))
    np.testing.assert_array_equal(got, z["bins"])


# Field at full, half and uneven resolution; offsets in y and x (z is unused, as in
# the reference); ranges that cut both values; bins of several shapes.
@pytest.mark.parametrize("vshape,fshape,offset,bins_shape,vrange,frange", [
    ((16, 32, 48), (16, 32, 48), (0, 0, 0), (32, 64), (1e4, 3e4), (1, 65535)),
    ((20, 36, 44), (10, 18, 22), (3, 5, 7), (64, 128), (1, 40000), (1, 65535)),
    ((21, 33, 45), (11, 17, 23), (0, 32, 0), (16, 256), (500.5, 20000.25), (1000, 50000)),
    ((9, 70, 300), (4, 35, 150), (0, 1, 299), (8, 8), (0, 65535), (0, 65535)),
    ((7, 13, 5), (3, 4, 2), (0, 0, 0), (1, 1), (100, 60000), (1, 65535)),
    ((12, 40, 40), (12, 40, 40), (0, 0, 0), (2048, 4096), (1, 30000), (1, 65535)),
])
def test_field_histogram_matches_oracle(vshape, fshape, offset, bins_shape, vrange, frange):
    rng = np.random.default_rng(sum(vshape) + sum(bins_shape))
    voxels = rng.integers(0, 65536, vshape, dtype=np.uint16)
    voxels[rng.random(vshape) < 0.2] = 0
    field = rng.integers(0, 65536, fshape, dtype=np.uint16)
    field[rng.random(fshape) < 0.1] = 0
    want = oracle.field_histogram(voxels, field, offset, bins_shape, vrange, frange)
    np.testing.assert_array_equal(_run(voxels, field, offset, bins_shape, vrange, frange), want)


def test_field_histogram_range_edges():
    """Voxel values on, just inside and just outside both ends of vrange."""
    vmin, vmax = 1000, 2000
    vals = np.array([0, 1, vmin - 1, vmin, vmin + 1, 1500, vmax - 1, vmax, vmax + 1, 65535], np.uint16)
    voxels = np.resize(vals, (4, 10, 30)).astype(np.uint16)
    field = np.resize(np.array([0, 1, 2, 65534, 65535, 30000], np.uint16), (4, 10, 30)).astype(np.uint16)
    for bins_shape in [(7, 11), (1, 1001), (65536 // 64, 64)]:
        want = oracle.field_histogram(voxels, field, (0, 0, 0), bins_shape, (vmin, vmax), (1, 65535))
        np.testing.assert_array_equal(_run(voxels, field, (0, 0, 0), bins_shape, (vmin, vmax), (1, 65535)), want)


def test_field_histogram_accumulates_into_bins():
    rng = np.random.default_rng(3)
    voxels = rng.integers(0, 40000, (8, 24, 24), dtype=np.uint16)
    field = rng.integers(0, 65536, (4, 12, 12), dtype=np.uint16)
    start = rng.integers(0, 1 << 40, (32, 32), dtype=np.uint64)
    want = start + oracle.field_histogram(voxels, field, (0, 0, 0), (32, 32), (1e4, 3e4), (1, 65535))
    np.testing.assert_array_equal(_run(voxels, field, (0, 0, 0), (32, 32), (1e4, 3e4), (1, 65535), start), want)


def test_field_histogram_contended_bin():
    """Every voxel lands in one bin: the warp-aggregated atomics must add up exactly."""
    voxels = torch.full((64, 256, 256), 15000, dtype=torch.int16, device="cuda")
    field = torch.full((32, 128, 128), 777, dtype=torch.int16, device="cuda")
    bins = torch.zeros((16, 16), dtype=torch.int64, device="cuda")
    field_histogram(voxels, field, (0, 0, 0), bins, (1e4, 3e4), (1, 65535), 0)
    got = bins.cpu().numpy()
    assert got.sum() == 64 * 256 * 256
    assert got[int(15 * (777 - 1) / 65534), int(15 * (5000 / 2e4))] == 64 * 256 * 256


def test_field_histogram_device_tensors_and_offset_past_the_end():
    rng = np.random.default_rng(5)
    voxels = rng.integers(0, 65536, (6, 20, 36), dtype=np.uint16)
    field = rng.integers(0, 65536, (3, 10, 18), dtype=np.uint16)
    tv = torch.from_numpy(voxels.view(np.int16)).cuda()
    tf = torch.from_numpy(field.view(np.int16)).cuda()
    bins = torch.zeros((32, 48), dtype=torch.int64, device="cuda")
    field_histogram(tv, tf, (0, 2, 3), bins, (1, 65535), (1, 65535), 0)
    want = oracle.field_histogram(voxels, field, (0, 2, 3), (32, 48), (1, 65535), (1, 65535))
    np.testing.assert_array_equal(bins.cpu().numpy().view(np.uint64), want)
    before = bins.clone()
    field_histogram(tv, tf, (0, 20, 0), bins, (1, 65535), (1, 65535), 0)  # y_start == nY: nothing to count
    field_histogram(tv, tf, (0, 0, 36), bins, (1, 65535), (1, 65535), 0)
    assert torch.equal(bins, before)


def test_field_histogram_rejects_bad_arguments():
    v = np.ones((2, 4, 4), np.uint16)
    f = np.ones((1, 2, 2), np.uint16)
    with pytest.raises(ValueError):
        field_histogram(v, f, (0, 0, 0), np.zeros((4, 4), np.uint64), (5, 5), (1, 65535), 0)
    with pytest.raises(ValueError):
        field_histogram(v, f, (0, -1, 0), np.zeros((4, 4), np.uint64), (1, 5), (1, 65535), 0)
    with pytest.raises(TypeError):
        field_histogram(v, f, (0, 0, 0), np.zeros((4, 4), np.int32), (1, 5), (1, 65535), 0)


def test_field_histogram_full_size_marginal():
    """512^3 voxels against a 256^3 field: summed over field bins, the histogram is the
    bincount of the voxel bins of every voxel whose field sample has a bin (torch FP64
    on the device, the reference's expressions)."""
    n = 512
    g = torch.Generator(device="cuda").manual_seed(11)
    voxels = torch.randint(0, 65536, (n, n, n), generator=g, device="cuda", dtype=torch.int32).to(torch.int16)
    field = torch.randint(0, 65536, (n // 2,) * 3, generator=g, device="cuda", dtype=torch.int32).to(torch.int16)
    vb_n, fb_n = 4096, 2048
    vmin, vmax, fmin, fmax = 1.0, 30000.0, 1.0, 65535.0
    bins = torch.zeros((fb_n, vb_n), dtype=torch.int64, device="cuda")
    field_histogram(voxels, field, (0, 0, 0), bins, (vmin, vmax), (fmin, fmax), 0)
    v = voxels.to(torch.int32) & 0xFFFF
    f = (field.to(torch.int32) & 0xFFFF).repeat_interleave(2, 0).repeat_interleave(2, 1).repeat_interleave(2, 2)
    vd = v.to(torch.float64)
    vd = torch.where((vd >= vmin) & (vd <= vmax), vd, torch.zeros_like(vd))
    vi = torch.floor((vb_n - 1) * ((vd - vmin) / (vmax - vmin))).to(torch.int64)
    fi = torch.floor((fb_n - 1) * ((f.to(torch.float64) - fmin) / (fmax - fmin))).to(torch.int64)
    keep = (vd != 0) & (f > 0) & (fi >= 0) & (fi < fb_n)
    want = torch.bincount(vi[keep], minlength=vb_n)
    assert torch.equal(bins.sum(0), want)
    assert torch.equal(bins.sum(1), torch.bincount(fi[keep], minlength=fb_n))
