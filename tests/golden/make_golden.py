"""Generate the golden vectors in this folder from the reference's own code.

Run where the reference tree is mounted and its CPU modules are built into
oracle/_ref (``make -C oracle ref``):

    python tests/golden/make_golden.py

Each case runs the reference pybind ``diffusion`` (OpenMP backend,
src/lib/cpp/cpu/diffusion.cc) on a seeded mask and kernel and stores the mask,
the float32 kernel, the repetition count and the uint16 result (plus its
sha256).  The bit-packing case stores the reference ``bitpacking.encode``
words for a seeded mask; the field-combination case stores two seeded uint16
fields and the result of the reference's 0975_combine_fields steps on them; the
histogram cases store a voxel volume, a field and the reference's
histograms.field_histogram bins, and a voxel block with the reference's
histograms.axis_histograms x / y / z / radial bins; the morphology case stores a
uint8 mask and the reference's morphology.dilate_3d_sphere / erode_3d_sphere results;
the implant case stores an implant mask, its frame of reference and the reference's
geometry.compute_front_back_masks outputs; the on-disk case stores a mask and the
uint8 file the reference CPU backend's on-disk overload writes for it
(``--on-disk`` regenerates only that case).  The tests then check the oracle bit-for-bit against
these files, and the CUDA library against the oracle.
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from maxibone_b200.kernels import gauss_kernel  # noqa: E402
from maxibone_b200.synthetic import spheres_mask  # noqa: E402


def test_kernel(sigma):
    """Kernel as the reference unit test builds it (src/test/test_diffusion.py:38-43)."""
    return gauss_kernel(sigma).astype(np.float32)


def cases():
    rng42 = np.random.RandomState(42)
    yield "reftest_n48_s3_r10", (rng42.rand(48, 48, 48) > 0.99).astype(np.uint8), test_kernel(3), 10
    yield "spheres_32x40x48_s2_r5", spheres_mask((32, 40, 48), 12, (3, 9), seed=1), test_kernel(2), 5
    yield "odd_17x23x41_s1.5_r3", (np.random.default_rng(2).random((17, 23, 41)) > 0.9).astype(np.uint8), \
        test_kernel(1.5), 3
    yield "thin_1x5x70_s3_r4", (np.random.default_rng(3).random((1, 5, 70)) > 0.8).astype(np.uint8), test_kernel(3), 4
    yield "wide_r_9x9x9_s4_r2", (np.random.default_rng(4).random((9, 9, 9)) > 0.7).astype(np.uint8), test_kernel(4), 2
    yield "zero_reps_8x8x8", (np.random.default_rng(5).random((8, 8, 8)) > 0.5).astype(np.uint8), test_kernel(1), 0
    yield "cfg0_128_spheres_s3_r10", spheres_mask((128, 128, 128), 40, (4, 20), seed=0), test_kernel(3), 10


def main():
    ref = oracle.reference_module("diffusion")
    bits = oracle.reference_module("bitpacking")
    if ref is None or bits is None:
        sys.exit("reference modules not built: run `make -C oracle ref` where the reference is mounted")
    index = {}
    for name, mask, kernel, reps in cases():
        out = np.empty(mask.shape, np.uint16)
        ref.diffusion(mask, kernel, out, reps)
        digest = hashlib.sha256(out.tobytes()).hexdigest()
        entry = {"shape": list(mask.shape), "kernel_size": int(kernel.shape[0]), "reps": reps, "sha256": digest}
        if mask.size <= 64 ** 3:
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), mask=mask, kernel=kernel,
                                reps=np.int64(reps), output=out)
            entry["file"] = f"{name}.npz"
        else:
            # Large case: the mask is regenerated from its seed; only the digest and a
            # middle slice are stored.
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), kernel=kernel, reps=np.int64(reps),
                                mask_sha256=np.bytes_(hashlib.sha256(mask.tobytes()).hexdigest()),
                                output_mid_slice=out[mask.shape[0] // 2])
            entry["file"] = f"{name}.npz"
            entry["mask"] = "spheres_mask((128,128,128), 40, (4, 20), seed=0)"
        index[name] = entry
        print(name, entry["sha256"][:16])
    m = (np.random.default_rng(7).random(32 * 32 * 8) > 0.5).astype(np.uint8)
    m[::7] = 3  # bit 0 set but not 1: the reference keeps `mask & 1`
    m[::11] = 2  # bit 0 clear
    packed = np.zeros(m.size // 32, np.uint32)
    bits.encode(m, packed, 0)
    decoded = np.zeros(m.size, np.uint8)
    bits.decode(packed, decoded, 0)
    np.savez_compressed(os.path.join(HERE, "bitpack_u32.npz"), mask=m, packed=packed, decoded=decoded)
    index["bitpack_u32"] = {"file": "bitpack_u32.npz", "n": int(m.size)}
    gen = oracle.reference_module("general")
    if gen is None:
        sys.exit("reference general module not built: run `make -C oracle ref`")
    # The Gaussian + EDT combination of src/processing_steps/0975_combine_fields.py:38-62:
    # its numpy steps, with to_int done by the reference's compiled normalized_convert.
    rng = np.random.default_rng(11)
    shape = (12, 48, 48)
    gauss = (rng.random(shape) ** 3 * 65535).astype(np.uint16)
    edt = (rng.random(shape) * 30000).astype(np.uint16)
    cylinder = oracle.cylinder_mask(shape[2])  # the script's generate_cylinder_mask(nx)
    combined = gauss.astype(np.float32) / gauss.max()
    combined -= edt.astype(np.float32) / edt.max()
    combined += np.abs(combined.min())
    combined /= combined.max()
    combined *= cylinder
    result = np.empty(shape, np.uint16)
    gen.normalized_convert(np.ascontiguousarray(combined), result)
    result *= cylinder
    np.savez_compressed(os.path.join(HERE, "combine_fields_u16.npz"), gauss=gauss, edt=edt, output=result)
    index["combine_fields_u16"] = {"file": "combine_fields_u16.npz", "shape": list(shape),
                                   "sha256": hashlib.sha256(result.tobytes()).hexdigest()}
    hist = oracle.reference_module("histograms")
    if hist is None:
        sys.exit("reference histograms module not built: run `make -C oracle ref`")
    # field_histogram of the histograms module (src/lib/cpp/cpu/histograms.cc:231-305) on
    # a voxel volume and a field at half its resolution, with the script's default ranges
    # (src/processing_steps/1000_compute_histograms.py:113).
    rng = np.random.default_rng(13)
    voxels = (rng.random((20, 36, 44)) * 40000).astype(np.uint16)
    field = (rng.random((10, 18, 22)) * 65535).astype(np.uint16)
    bins = np.zeros((64, 128), np.uint64)
    hist.field_histogram(voxels, field, (0, 0, 0), bins, (1e4, 3e4), (1, 2 ** 16 - 1), 0)
    np.savez_compressed(os.path.join(HERE, "field_histogram_u64.npz"), voxels=voxels, field=field, bins=bins,
                        vrange=np.array([1e4, 3e4]), frange=np.array([1.0, 2.0 ** 16 - 1]))
    index["field_histogram_u64"] = {"file": "field_histogram_u64.npz", "bins": list(bins.shape),
                                    "total": int(bins.sum())}
    # axis_histograms (src/lib/cpp/cpu/histograms.cc:14-80) on a z-block of a volume, as
    # the out-of-core loop calls it (src/processing_steps/1000_compute_histograms.py:470),
    # with the script's centre and radial extent (:60-62).
    gshape, z_start = (40, 36, 44), 16
    block = rng.integers(0, 40000, (16, 36, 44), dtype=np.uint16)
    block[rng.random(block.shape) < 0.15] = 0
    center = (gshape[1] // 2, gshape[2] // 2)
    n_r = int(np.sqrt((gshape[2] // 2) ** 2 + (gshape[1] // 2) ** 2)) + 1
    xb, yb = np.zeros((gshape[2], 256), np.uint64), np.zeros((gshape[1], 256), np.uint64)
    zb, rb = np.zeros((gshape[0], 256), np.uint64), np.zeros((n_r, 256), np.uint64)
    hist.axis_histograms(block, (z_start, 0, 0), xb, yb, zb, rb, center, (1e4, 3e4), 0)
    np.savez_compressed(os.path.join(HERE, "axis_histograms_u64.npz"), voxels=block, z_start=z_start,
                        global_shape=np.array(gshape), center=np.array(center), vrange=np.array([1e4, 3e4]),
                        x_bins=xb, y_bins=yb, z_bins=zb, r_bins=rb)
    index["axis_histograms_u64"] = {"file": "axis_histograms_u64.npz", "voxel_bins": 256, "n_r": n_r,
                                    "total": int(xb.sum())}
    morph = oracle.reference_module("morphology")
    if morph is None:
        sys.exit("reference morphology module not built: run `make -C oracle ref`")
    # dilate_3d_sphere / erode_3d_sphere (src/lib/cpp/cpu_seq/morphology.cc:14-99) on a
    # seeded sphere mask with a few stray voxels, one of them a byte with bit 0 clear
    # (erosion reads bit 0 only); radius 16 takes the reference's dedicated r16 path.
    mshape = (24, 32, 72)
    mmask = spheres_mask(mshape, 14, (3, 10), seed=4)
    mmask = np.maximum(mmask, (np.random.default_rng(4).random(mshape) > 0.997).astype(np.uint8))
    mmask[12, 16, 30] = 2
    results = {}
    for name, fn, r in [("dilate_r3", morph.dilate_3d_sphere, 3), ("dilate_r16", morph.dilate_3d_sphere, 16),
                        ("erode_r2", morph.erode_3d_sphere, 2), ("erode_r5", morph.erode_3d_sphere, 5)]:
        res = np.zeros(mshape, np.uint8)
        fn(mmask, r, res)
        results[name] = res
    np.savez_compressed(os.path.join(HERE, "morphology_u8.npz"), mask=mmask, **results)
    index["morphology_u8"] = {"file": "morphology_u8.npz", "shape": list(mshape),
                              "counts": {k: int(v.sum()) for k, v in results.items()}}
    geo = oracle.reference_module("geometry")
    if geo is None:
        sys.exit("reference geometry module not built: run `make -C oracle ref`")
    # compute_front_back_masks (src/lib/cpp/cpu_seq/geometry.cc:112-215) on a tilted
    # cylinder with stray voxels, a rotation E, a second rotation UVWp and an offset cp,
    # as src/processing_steps/0750_bone_region.py:62 passes them (float64, cast by the binding).
    ishape = (28, 40, 44)
    irng = np.random.default_rng(17)
    zz, yy, xx = np.meshgrid(*(np.arange(n) for n in ishape), indexing="ij")
    implant = ((((yy - 21.0 - 0.2 * zz) ** 2 + (xx - 20.5) ** 2) < 64.0) & (zz > 2)).astype(np.uint8)
    implant[irng.random(ishape) > 0.999] = 1
    E = np.linalg.qr(irng.normal(size=(3, 3)))[0]
    UVWp = np.linalg.qr(irng.normal(size=(3, 3)))[0]
    cm = np.array(np.nonzero(implant)).mean(axis=1)
    cp = irng.normal(size=3) * 4
    voxel_size = 1.875
    outs = [np.empty(ishape, np.uint8) for _ in range(4)]
    geo.compute_front_back_masks(implant, voxel_size, E, cm, cp, UVWp, *outs)
    np.savez_compressed(os.path.join(HERE, "implant_masks_u8.npz"), mask=implant, E=E, cm=cm, cp=cp, UVWp=UVWp,
                        voxel_size=np.array(voxel_size), front=outs[0], back=outs[1], shell=outs[2], solid=outs[3])
    index["implant_masks_u8"] = {"file": "implant_masks_u8.npz", "shape": list(ishape),
                                 "counts": {k: int(v.sum()) for k, v in zip(("front", "back", "shell", "solid"), outs)}}
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


def on_disk_case():
    """The reference CPU backend's on-disk overload, diffusion(input_file,
    np_kernel, output_file, total_shape, global_shape, repititions)
    (src/pybind/diffusion-pybind.cc:67-77, src/lib/cpp/cpu/diffusion.cc:376-468):
    a raw uint8 mask file in, a raw uint8 file of floor(v * 255) out, computed in
    z-blocks of global_shape[0] planes with the mask rebuilt as field == 1.0f
    before every repetition.  The block depth leaves a partial last block.  The
    reference keeps its float temporaries in /tmp/maxibone (a path fixed in its
    source); they are removed afterwards."""
    import shutil
    import tempfile

    ref = oracle.reference_module("diffusion")
    if ref is None:
        sys.exit("reference modules not built: run `make -C oracle ref`")
    shape, global_z, reps = (40, 24, 32), 12, 4
    mask = spheres_mask(shape, 10, (2, 7), seed=21)
    kernel = test_kernel(1.5)
    temp_existed = os.path.exists("/tmp/maxibone")
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "mask.uint8"), os.path.join(d, "field.uint8")
        mask.tofile(fin)
        ref.diffusion(fin, kernel, fout, shape, (global_z, shape[1], shape[2]), reps, 0)
        out = np.fromfile(fout, dtype=np.uint8).reshape(shape)
    if not temp_existed:
        shutil.rmtree("/tmp/maxibone", ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, "on_disk_cpu_u8.npz"), mask=mask, kernel=kernel, reps=np.int64(reps),
                        global_z=np.int64(global_z), output=out)
    with open(os.path.join(HERE, "index.json")) as f:
        index = json.load(f)
    index["on_disk_cpu_u8"] = {"file": "on_disk_cpu_u8.npz", "shape": list(shape), "global_z": global_z,
                               "reps": reps, "sha256": hashlib.sha256(out.tobytes()).hexdigest()}
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)
    print("on_disk_cpu_u8", index["on_disk_cpu_u8"]["sha256"][:16])


if __name__ == "__main__":
    if "--on-disk" in sys.argv:
        on_disk_case()
    else:
        main()
        on_disk_case()
