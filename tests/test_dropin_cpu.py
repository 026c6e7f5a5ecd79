"""The drop-in ``diffusion`` mirrors the reference pybind conversions
(src/pybind/diffusion-pybind.cc:81-85) -- checked without a GPU."""
import numpy as np
import pytest

from maxibone_b200 import diffusion, gauss_kernel
from maxibone_b200._lib import MaxiError


def test_output_is_not_converted():
    m = np.zeros((4, 4, 4), np.uint8)
    k = gauss_kernel(1)
    for bad in [np.zeros((4, 4, 4), np.int32), np.zeros((4, 4, 4), np.uint16)[:, :, ::-1], [[0]]]:
        with pytest.raises(TypeError):
            diffusion(m, k, bad, 1)


def test_shape_checks_raise_value_error():
    k = gauss_kernel(1)
    with pytest.raises(ValueError):
        diffusion(np.zeros((4, 4), np.uint8), k, np.zeros((4, 4), np.uint16))
    with pytest.raises(ValueError):
        diffusion(np.zeros((4, 4, 4), np.uint8), k, np.zeros((4, 4, 5), np.uint16))
    with pytest.raises(ValueError):
        diffusion(np.zeros((4, 4, 4), np.uint8), np.ones(4), np.zeros((4, 4, 4), np.uint16))


def test_repititions_must_be_int():
    with pytest.raises(TypeError):
        diffusion(np.zeros((4, 4, 4), np.uint8), gauss_kernel(1), np.zeros((4, 4, 4), np.uint16), 1.5)


def test_forcecast_inputs_reach_the_library():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible; the GPU tests cover the call")
    # bool mask and float64 kernel are converted like pybind's forcecast; with no
    # GPU the library reports that instead of computing on the CPU.
    with pytest.raises(MaxiError, match="NO_DEVICE"):
        diffusion(np.zeros((4, 4, 4), bool), gauss_kernel(1), np.zeros((4, 4, 4), np.uint16), repititions=2)


def test_gauss_kernel_matches_reference_construction():
    # src/test/test_diffusion.py:38-43 / src/lib/py/helpers.py:402-408
    sigma = 3
    radius = round(4.0 * sigma)
    x = np.arange(-radius, radius + 1)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    np.testing.assert_array_equal(gauss_kernel(sigma), phi / phi.sum())
    assert gauss_kernel(8).shape == (65,)
    assert gauss_kernel(32).shape == (257,)


def test_on_disk_overload_io_errors_without_gpu(tmp_path):
    from maxibone_b200._lib import MaxiError
    with pytest.raises(MaxiError, match="IO"):
        diffusion(str(tmp_path / "missing.uint8"), gauss_kernel(1), str(tmp_path / "out.uint16"),
                  (4, 4, 4), (2, 4, 4), 1)
    short = tmp_path / "short.uint8"
    np.zeros(10, np.uint8).tofile(short)
    with pytest.raises(MaxiError, match="fewer than"):
        diffusion(str(short), gauss_kernel(1), str(tmp_path / "out.uint16"), (4, 4, 4), (2, 4, 4), 1)
    with pytest.raises(ValueError):
        diffusion(str(short), gauss_kernel(1), str(tmp_path / "out.uint16"), (4, 4), (2, 4, 4), 1)
