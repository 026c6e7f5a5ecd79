"""Pins the CPU oracle (the parity checker) against the reference.

* golden vectors made by the reference's own OpenMP module (tests/golden);
* the reference module itself where it has been built into oracle/_ref;
* the scipy chain of the reference's unit test (src/test/test_diffusion.py:49-98),
  with its 1-LSB criterion, at the test's own configuration.
"""
import hashlib

import numpy as np
import pytest

import oracle
from conftest import DIFFUSION_CASES, load_golden
from maxibone_b200.kernels import gauss_kernel


@pytest.mark.parametrize("name", DIFFUSION_CASES)
def test_oracle_matches_reference_golden_bit_for_bit(name):
    mask, kernel, reps, out, entry = load_golden(name)
    got, _ = oracle.diffusion_in_memory(mask, kernel, reps)
    assert hashlib.sha256(got.tobytes()).hexdigest() == entry["sha256"]
    if out is not None:
        np.testing.assert_array_equal(got, out)


def test_oracle_bitpack_matches_reference_golden():
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "bitpack_u32.npz"))
    np.testing.assert_array_equal(oracle.bitpack_encode(z["mask"]), z["packed"])
    np.testing.assert_array_equal(oracle.bitpack_decode(z["packed"], z["mask"].size), z["decoded"])


def test_oracle_matches_reference_module_if_built():
    ref = oracle.reference_module()
    if ref is None:
        pytest.skip("reference module not built in oracle/_ref")
    rng = np.random.default_rng(11)
    for shape, sigma, reps in [((20, 31, 44), 2.0, 3), ((3, 64, 5), 3.0, 2), ((40, 1, 40), 1.0, 6)]:
        mask = (rng.random(shape) > 0.85).astype(np.uint8)
        k = gauss_kernel(sigma).astype(np.float32)
        want = np.empty(shape, np.uint16)
        ref.diffusion(mask, k, want, reps)
        got, _ = oracle.diffusion_in_memory(mask, k, reps)
        np.testing.assert_array_equal(got, want)


def test_reference_unit_test_configuration_scipy_within_1_lsb():
    # src/test/test_diffusion.py:19-43: n=128, sigma=3, reps=100, seed 42, rand > 0.99.
    np.random.seed(42)
    a = np.random.rand(128, 128, 128) > 0.99
    kernel = gauss_kernel(3).astype(np.float32)
    want = oracle.scipy_chain(a, kernel, 100)
    got, _ = oracle.diffusion_in_memory(a.astype(np.uint8), kernel, 100)
    assert np.abs(want.astype(np.int32) - got.astype(np.int32)).max() <= 1


def test_f64_oracle_close_to_f32_oracle():
    rng = np.random.default_rng(5)
    mask = (rng.random((24, 30, 36)) > 0.9).astype(np.uint8)
    k = gauss_kernel(2.0)
    f64 = oracle.diffusion_f64(mask, k, 8)
    _, f32 = oracle.diffusion_in_memory(mask, k.astype(np.float32), 8)
    assert np.abs(f64 - f32).max() < 2e-6


def test_on_disk_semantics_equal_in_memory_for_binary_field():
    # The on-disk variant rebuilds the mask as field == 1.0f; with no non-mask voxel
    # reaching exactly 1.0 the two agree.
    rng = np.random.default_rng(6)
    mask = (rng.random((16, 18, 20)) > 0.95).astype(np.uint8)
    k = gauss_kernel(1.0).astype(np.float32)
    a = oracle.diffusion_on_disk_semantics(mask, k, 4)
    b, _ = oracle.diffusion_in_memory(mask, k, 4)
    np.testing.assert_array_equal(a, b)


def test_oracle_combine_fields_matches_reference_golden():
    # src/processing_steps/0975_combine_fields.py:38-62 with the reference's compiled to_int.
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "combine_fields_u16.npz"))
    np.testing.assert_array_equal(oracle.combine_fields(z["gauss"], z["edt"]), z["output"])


def test_oracle_normalized_convert_matches_reference_module():
    gen = oracle.reference_module("general")
    if gen is None:
        pytest.skip("reference general module not built (make -C oracle ref)")
    rng = np.random.default_rng(3)
    for shape in [(3, 5, 7), (8, 33, 40)]:
        x = (rng.standard_normal(shape) * 3).astype(np.float32)
        want = np.empty(shape, np.uint16)
        gen.normalized_convert(x, want)
        np.testing.assert_array_equal(oracle.normalized_convert_u16(x), want)


def test_oracle_cylinder_mask_square_and_general():
    m = oracle.cylinder_mask(48)
    assert m.shape == (48, 48) and m.dtype == bool
    assert not m[0, 0] and m[24, 24]
    assert oracle.cylinder_mask(1, 5).sum() == 0  # linspace(-1, 1, 1) == [-1]: nothing inside
    assert oracle.cylinder_mask(10, 20).shape == (10, 20)


def test_oracle_field_histogram_matches_reference_golden():
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "field_histogram_u64.npz"))
    got = oracle.field_histogram(z["voxels"], z["field"], (0, 0, 0), z["bins"].shape, tuple(z["vrange"]),
                                 tuple(z["frange"]))
    np.testing.assert_array_equal(got, z["bins"])


def test_oracle_field_histogram_matches_reference_module_with_offsets():
    hist = oracle.reference_module("histograms")
    if hist is None:
        pytest.skip("reference histograms module not built (make -C oracle ref)")
    rng = np.random.default_rng(5)
    v = rng.integers(0, 65535, (9, 17, 23), dtype=np.uint16)
    f = rng.integers(0, 65535, (5, 9, 12), dtype=np.uint16)
    want = np.zeros((40, 70), np.uint64)
    hist.field_histogram(v, f, (0, 3, 5), want, (0.0, 65535.0), (1.0, 65535.0), 0)
    np.testing.assert_array_equal(oracle.field_histogram(v, f, (0, 3, 5), (40, 70), (0.0, 65535.0), (1.0, 65535.0)),
                                  want)


def test_oracle_axis_histograms_matches_reference_golden():
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "axis_histograms_u64.npz"))
    got = oracle.axis_histograms(z["voxels"], (int(z["z_start"]), 0, 0), tuple(z["global_shape"]),
                                 z["x_bins"].shape[1], z["r_bins"].shape[0], tuple(z["center"]), tuple(z["vrange"]))
    for g, name in zip(got, ("x_bins", "y_bins", "z_bins", "r_bins")):
        np.testing.assert_array_equal(g, z[name], err_msg=name)


@pytest.mark.parametrize("zoff,yoff,xoff,center,nzb", [(0, 0, 0, (20, 25), 30), (10, 3, 7, (20, 25), 12),
                                                         (25, 0, 0, (5, 44), 12)])
def test_oracle_axis_histograms_matches_reference_module(zoff, yoff, xoff, center, nzb):
    """Offsets in every axis, an off-centre centre and a block that runs past Nz."""
    hist = oracle.reference_module("histograms")
    if hist is None:
        pytest.skip("reference histograms module not built (make -C oracle ref)")
    gs, nb, vr = (30, 40, 50), 64, (500.5, 3e4)
    rng = np.random.default_rng(zoff + nzb)
    v = rng.integers(0, 40000, (nzb, gs[1], gs[2]), dtype=np.uint16)
    n_r = int(np.ceil(np.hypot(max(center[0], gs[1] - center[0]), max(center[1], gs[2] - center[1])))) + 1
    want = (np.zeros((gs[2], nb), np.uint64), np.zeros((gs[1], nb), np.uint64), np.zeros((gs[0], nb), np.uint64),
            np.zeros((n_r, nb), np.uint64))
    hist.axis_histograms(v, (zoff, yoff, xoff), *want, center, vr, 0)
    got = oracle.axis_histograms(v, (zoff, yoff, xoff), gs, nb, n_r, center, vr)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def _golden_morph():
    import os
    from conftest import GOLDEN
    return np.load(os.path.join(GOLDEN, "morphology_u8.npz"))


def test_oracle_morphology_matches_reference_golden():
    z = _golden_morph()
    for name in ("dilate_r3", "dilate_r16", "erode_r2", "erode_r5"):
        op, r = name.split("_r")
        np.testing.assert_array_equal(oracle.morphology_sphere(z["mask"], int(r), op == "dilate"), z[name],
                                      err_msg=name)


@pytest.mark.parametrize("r", [0, 1, 4, 7, 15])
def test_oracle_morphology_bitpacked_equals_packed_reference_for_small_radii(r):
    """Below radius 16 the bit-packed kernel rows hold the whole sphere, so the packed
    form equals the reference's uint8 result packed (MSB first)."""
    z = _golden_morph()
    m = np.ascontiguousarray(z["mask"][:, :, :64])  # whole words
    words = np.packbits((m != 0).astype(np.uint8), axis=-1).view(">u4").astype(np.uint32).reshape(
        m.shape[0], m.shape[1], -1)
    got = oracle.morphology_sphere_bitpacked(words, r, True)
    want = np.packbits(oracle.morphology_sphere(m, r, True), axis=-1).view(">u4").astype(np.uint32).reshape(
        words.shape)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("shape,r", [((9, 10, 11), 0), ((12, 14, 16), 1), ((20, 22, 24), 5), ((18, 20, 37), 16),
                                     ((8, 30, 40), 9)])
def test_oracle_morphology_matches_reference_module(shape, r):
    morph = oracle.reference_module("morphology")
    if morph is None:
        pytest.skip("reference morphology module not built (make -C oracle ref)")
    rng = np.random.default_rng(r + shape[2])
    m = (rng.random(shape) > 0.4).astype(np.uint8)
    m[rng.random(shape) > 0.97] = 2
    for dilate, fn in ((True, morph.dilate_3d_sphere), (False, morph.erode_3d_sphere)):
        want = np.zeros(shape, np.uint8)
        fn(m, r, want)
        np.testing.assert_array_equal(oracle.morphology_sphere(m, r, dilate), want)


def test_oracle_implant_masks_match_reference_golden():
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "implant_masks_u8.npz"))
    got = oracle.implant_masks(z["mask"], float(z["voxel_size"]), z["E"], z["cm"], z["cp"], z["UVWp"])
    for g, name in zip(got, ("front", "back", "shell", "solid")):
        np.testing.assert_array_equal(g, z[name], err_msg=name)


@pytest.mark.parametrize("seed,shape", [(1, (24, 40, 48)), (2, (33, 31, 29)), (3, (16, 64, 64))])
def test_oracle_implant_masks_match_reference_module(seed, shape):
    geo = oracle.reference_module("geometry")
    if geo is None:
        pytest.skip("reference geometry module not built (make -C oracle ref)")
    rng = np.random.default_rng(seed)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    implant = ((((yy - ny / 2 - 2) ** 2 + (xx - nx / 2 + 1) ** 2) < (min(ny, nx) / 4) ** 2) & (zz > 3)).astype(np.uint8)
    implant[rng.random(shape) > 0.999] = 1
    implant[rng.random(shape) > 0.9995] = 3  # a byte other than 1: mask & and | act on its bits
    E = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    UVWp = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    cm = np.array(np.nonzero(implant)).mean(axis=1)
    cp = rng.normal(size=3) * 5
    want = [np.empty(shape, np.uint8) for _ in range(4)]
    geo.compute_front_back_masks(implant, 1.875, E, cm, cp, UVWp, *want)
    for g, w in zip(oracle.implant_masks(implant, 1.875, E, cm, cp, UVWp), want):
        np.testing.assert_array_equal(g, w)


def test_on_disk_semantics_pinned_to_the_reference_cpu_on_disk_overload():
    # The reference CPU backend's on-disk overload (z-blocks with radius halos,
    # mask rebuilt as field == 1.0f every repetition, float temporaries on disk)
    # writes (uint8) floor(v * 255); the oracle's whole-volume restatement of the
    # same semantics, converted the same way, must equal that file bit for bit.
    import os
    from conftest import GOLDEN
    z = np.load(os.path.join(GOLDEN, "on_disk_cpu_u8.npz"))
    got = oracle.diffusion_on_disk_u8(z["mask"], z["kernel"], int(z["reps"]))
    np.testing.assert_array_equal(got, z["output"])
