"""The field histogram (src/lib/cpp/cpu/histograms.cc:231-305 via
src/pybind/histograms-pybind.cc:81-107) and the axis histograms (histograms.cc:14-80
via histograms-pybind.cc:30-66) on the GPU against their oracles and the goldens
made by the reference's own module (run with -m gpu).  Counts are
integers from the reference's FP64 bin expressions, so they must be identical."""
import os

import numpy as np
import pytest
import torch

import oracle
from conftest import GOLDEN
from maxibone_b200.histograms import axis_histograms, field_histogram

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
    ((8, 24, 64), (4, 12, 32), (0, 3, 13), (128, 512), (1, 40000), (1, 65535)),
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


# Every uint16 value through the voxel and field bin maps: ranges narrower than the
# bin count (bins with no value), a high vmin with a tiny span, fractional bounds,
# a single bin, one bin per value, and the full range.
@pytest.mark.parametrize("lo,hi,nbins", [(1e4, 3e4, 4096), (60000, 60010, 4096), (0.5, 65535.5, 65536),
                                         (123.25, 40000.75, 2048), (1, 65535, 1), (0, 65535, 65535),
                                         (65000, 65535, 7), (2.0, 3.0, 1000)])
def test_bin_maps_cover_every_value(lo, hi, nbins):
    every = np.arange(65536, dtype=np.uint16).reshape(16, 64, 64)
    same = np.full(every.shape, 40000, np.uint16)
    # voxel map: every value against one counted field value
    want = oracle.field_histogram(every, same, (0, 0, 0), (4, nbins), (lo, hi), (1, 65535))
    np.testing.assert_array_equal(_run(every, same, (0, 0, 0), (4, nbins), (lo, hi), (1, 65535)), want)
    # field map: one counted voxel value against every field value
    want = oracle.field_histogram(same, every, (0, 0, 0), (nbins, 4), (1, 65535), (lo, hi))
    np.testing.assert_array_equal(_run(same, every, (0, 0, 0), (nbins, 4), (1, 65535), (lo, hi)), want)
    # axis histograms: every value in every row and column position
    gs = every.shape
    n_r = int(np.ceil(np.hypot(32, 32))) + 1
    want = oracle.axis_histograms(every, (0, 0, 0), gs, nbins, n_r, (32, 32), (lo, hi))
    got = _axis_run(every, (0, 0, 0), gs, nbins, n_r, (32, 32), (lo, hi))
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


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


def _axis_run(voxels, offset, gshape, voxel_bins, n_r, center, vrange):
    out = (np.zeros((gshape[2], voxel_bins), np.uint64), np.zeros((gshape[1], voxel_bins), np.uint64),
           np.zeros((gshape[0], voxel_bins), np.uint64), np.zeros((n_r, voxel_bins), np.uint64))
    axis_histograms(voxels, offset, *out, center, vrange, 0)
    return out


def test_axis_histograms_matches_reference_golden():
    z = np.load(os.path.join(GOLDEN, "axis_histograms_u64.npz"))
    got = _axis_run(z["voxels"], (int(z["z_start"]), 0, 0), tuple(z["global_shape"]), z["x_bins"].shape[1],
                    z["r_bins"].shape[0], tuple(int(c) for c in z["center"]), tuple(z["vrange"]))
    for g, name in zip(got, ("x_bins", "y_bins", "z_bins", "r_bins")):
        np.testing.assert_array_equal(g, z[name], err_msg=name)


# Blocks at several z offsets (one past Nz), y / x offsets, centres off the middle and
# at a corner (radii past n_r are skipped), rows wider than a block of threads.
@pytest.mark.parametrize("gshape,nzb,offset,center,voxel_bins,vrange,n_r", [
    ((30, 40, 50), 30, (0, 0, 0), (20, 25), 64, (1e4, 3e4), None),
    ((30, 40, 50), 12, (10, 3, 7), (20, 25), 128, (1, 40000), None),
    ((30, 40, 50), 12, (25, 0, 0), (5, 44), 32, (500.5, 2e4), None),
    ((9, 33, 17), 9, (0, 0, 0), (16, 8), 1, (0, 65535), None),
    ((6, 20, 600), 6, (0, 2, 300), (0, 0), 256, (1, 65535), 100),
    ((4, 64, 64), 4, (0, 0, 0), (32, 32), 4096, (1, 32000), 46),
])
def test_axis_histograms_matches_oracle(gshape, nzb, offset, center, voxel_bins, vrange, n_r):
    if n_r is None:
        n_r = int(np.ceil(np.hypot(max(center[0], gshape[1] - center[0]), max(center[1], gshape[2] - center[1])))) + 1
    rng = np.random.default_rng(sum(gshape) + nzb + voxel_bins)
    voxels = rng.integers(0, 40000, (nzb, gshape[1], gshape[2]), dtype=np.uint16)
    voxels[rng.random(voxels.shape) < 0.2] = 0
    want = oracle.axis_histograms(voxels, offset, gshape, voxel_bins, n_r, center, vrange)
    got = _axis_run(voxels, offset, gshape, voxel_bins, n_r, center, vrange)
    for g, w, name in zip(got, want, ("x", "y", "z", "r")):
        np.testing.assert_array_equal(g, w, err_msg=name)


def test_axis_histograms_device_tensors_accumulate():
    """Two z-blocks of one volume added into the same device bins equal one pass over the
    volume (the out-of-core loop of the histogram step)."""
    gshape, vb, center = (24, 48, 40), 128, (24, 20)
    n_r = int(np.sqrt(20 ** 2 + 24 ** 2)) + 1
    rng = np.random.default_rng(8)
    vol = rng.integers(0, 65536, gshape, dtype=np.uint16)
    bins = [torch.zeros((n, vb), dtype=torch.int64, device="cuda") for n in (gshape[2], gshape[1], gshape[0], n_r)]
    for z0 in (0, 10):
        blk = torch.from_numpy(np.ascontiguousarray(vol[z0:z0 + 14]).view(np.int16)).cuda()
        axis_histograms(blk, (z0, 0, 0), *bins, center, (1, 65535), 0)
    want = oracle.axis_histograms(vol, (0, 0, 0), gshape, vb, n_r, center, (1, 65535))
    # planes 10..13 are in both blocks
    extra = oracle.axis_histograms(vol[10:14], (10, 0, 0), gshape, vb, n_r, center, (1, 65535))
    for b, w, e in zip(bins, want, extra):
        np.testing.assert_array_equal(b.cpu().numpy().view(np.uint64), w + e)


def test_axis_histograms_rejects_bad_arguments():
    v = np.ones((2, 4, 6), np.uint16)
    xb, yb, zb, rb = (np.zeros((n, 8), np.uint64) for n in (6, 4, 2, 5))
    with pytest.raises(ValueError):  # voxel block rows must match len(y_bins), len(x_bins)
        axis_histograms(np.ones((2, 4, 5), np.uint16), (0, 0, 0), xb, yb, zb, rb, (2, 3), (1, 5), 0)
    with pytest.raises(ValueError):
        axis_histograms(v, (0, 0, 0), xb, yb, zb, np.zeros((5, 9), np.uint64), (2, 3), (1, 5), 0)
    with pytest.raises(ValueError):
        axis_histograms(v, (0, 0, 0), xb, yb, zb, rb, (2, 3), (5, 1), 0)
    with pytest.raises(TypeError):
        axis_histograms(v, (0, 0, 0), xb, yb, zb, rb, (-1, 3), (1, 5), 0)


def test_axis_histograms_full_size_marginals():
    """A 256-plane block of a 1024^2-plane volume: every histogram sums to the number of
    counted voxels, and the z rows equal per-plane bincounts (torch FP64 on the device)."""
    n, nzb, vb = 1024, 256, 4096
    g = torch.Generator(device="cuda").manual_seed(2)
    vox = torch.randint(0, 40000, (nzb, n, n), generator=g, device="cuda", dtype=torch.int32)
    n_r = int(np.sqrt(2 * (n // 2) ** 2)) + 1
    bins = [torch.zeros((k, vb), dtype=torch.int64, device="cuda") for k in (n, n, 2 * nzb, n_r)]
    axis_histograms(vox.to(torch.int16), (nzb, 0, 0), *bins, (n // 2, n // 2), (1.0, 32000.0), 0)
    vd = vox.to(torch.float64)
    vd = torch.where((vd >= 1.0) & (vd <= 32000.0), vd, torch.zeros_like(vd))
    vi = torch.floor((vb - 1) * ((vd - 1.0) / 31999.0)).to(torch.int64)
    keep = vd != 0
    total = int(keep.sum())
    for b in bins:
        assert int(b.sum()) == total
    want_z = torch.stack([torch.bincount(vi[z][keep[z]], minlength=vb) for z in range(nzb)])
    assert torch.equal(bins[2][nzb:], want_z) and int(bins[2][:nzb].sum()) == 0
