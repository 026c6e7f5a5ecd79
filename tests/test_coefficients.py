"""The single 16-bit coefficient set of the tensor-core passes (CPU: the set is
chosen on the host, read through maxi_tensor_core_taps).

Plainly rounded BF16 taps miss the kernel's sum by ~1e-4 (3e-5 at best for
sigma 2 at any one scale), and that gain error compounds over the 3 R passes of
a diffusion.  The passes therefore search the scale of the set: its taps times
the factor their epilogues apply must keep the FP32 kernel's sum (to 2e-7 at
sigma 1, 2e-8 from sigma 2; ~1e-9 for most sigmas) and
its second moment closely, and stay symmetric."""
import ctypes

import numpy as np
import pytest

from maxibone_b200 import _lib, gauss_kernel


def taps_of(kernel, field):
    k = np.ascontiguousarray(kernel, np.float32)
    bits = np.zeros(k.size, np.uint16)
    inv = ctypes.c_float()
    _lib.check(_lib.lib().maxi_tensor_core_taps(k.ctypes.data, k.size, _lib.FIELD_TYPES[field], bits.ctypes.data,
                                                ctypes.byref(inv)))
    if field == "bf16":
        values = (bits.astype(np.uint32) << 16).view(np.float32).astype(np.float64)
    else:
        values = bits.view(np.float16).astype(np.float64)
    return values, float(inv.value)


@pytest.mark.parametrize("field", ["bf16", "f16"])
@pytest.mark.parametrize("sigma", [1.0, 2.0, 3.0, 4.0, 6.0, 8.0, 16.0])
def test_scaled_set_keeps_sum_and_second_moment(field, sigma):
    kernel = gauss_kernel(sigma).astype(np.float32)
    r = kernel.size // 2
    values, inv = taps_of(kernel, field)
    eff = values * inv  # what a pass multiplies the field by
    k64 = kernel.astype(np.float64)
    j2 = (np.arange(-r, r + 1, dtype=np.float64)) ** 2
    assert abs(eff.sum() - k64.sum()) < (2e-7 if sigma < 2 else 2e-8)
    assert abs((j2 * eff).sum() - (j2 * k64).sum()) < 1e-3 * max(1.0, (j2 * k64).sum())
    np.testing.assert_array_equal(values, values[::-1])  # symmetric kernel, symmetric taps
    # each tap is one of the two 16-bit neighbours of the scaled FP32 tap
    assert np.all(np.abs(values - k64 / inv) <= np.abs(k64 / inv) * (2.0 ** -7 if field == "bf16" else 2.0 ** -10)
                  + 1e-30)


def test_plain_rounding_would_miss_the_sum():
    # the reason for the search: sigma 2 with round-to-nearest BF16 taps
    kernel = gauss_kernel(2.0).astype(np.float32)
    bits = kernel.view(np.uint32)
    rounded = ((bits.astype(np.uint64) + 0x7FFF + ((bits >> 16) & 1)) >> 16) << 16  # round to nearest even
    plain = rounded.astype(np.uint32).view(np.float32).astype(np.float64)
    assert abs(plain.sum() - kernel.astype(np.float64).sum()) > 1e-5
    values, inv = taps_of(kernel, "bf16")
    assert abs((values * inv).sum() - kernel.astype(np.float64).sum()) < 1e-7


@pytest.mark.parametrize("size,field", [(4, "bf16"), (259, "bf16"), (5, "f32")])
def test_rejects_bad_arguments(size, field):
    k = np.ones(size, np.float32) / size
    bits = np.zeros(size, np.uint16)
    inv = ctypes.c_float()
    rc = _lib.lib().maxi_tensor_core_taps(k.ctypes.data, size, _lib.FIELD_TYPES[field], bits.ctypes.data,
                                          ctypes.byref(inv))
    assert rc == 1  # MAXI_ERR_INVALID_ARGUMENT
