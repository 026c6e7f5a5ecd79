"""Generate the golden vectors in this folder from the reference's own code.

Run where the reference tree is mounted and its CPU modules are built into
oracle/_ref (``make -C oracle ref``):

    python tests/golden/make_golden.py

Each case runs the reference pybind ``diffusion`` (OpenMP backend,
src/lib/cpp/cpu/diffusion.cc) on a seeded mask and kernel and stores the mask,
the float32 kernel, the repetition count and the uint16 result (plus its
sha256).  The bit-packing case stores the reference ``bitpacking.encode``
words for a seeded mask; the field-combination case stores two seeded uint16
fields and the result of the reference's 0975_combine_fields steps on them.  The tests then check the oracle bit-for-bit against
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
    with open(os.path.join(HERE, "index.json"), "w") as f:
        json.dump(index, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
