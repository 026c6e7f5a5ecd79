"""1-D Gaussian kernels for the diffusion path."""
from __future__ import annotations

import numpy as np


def gauss_kernel(sigma: float) -> np.ndarray:
    """Normalised 1-D Gaussian in FP64, radius round(4*sigma).

    Same construction as the reference's ``gauss_kernel``
    (src/lib/py/helpers.py:376-409), which follows scipy's gaussian_filter1d:
    x = -r..r, phi = exp(-0.5 / sigma^2 * x^2), phi / sum(phi).
    The diffusion call casts it to float32, as pybind's forcecast does.
    """
    if sigma <= 0:
        raise ValueError("sigma must be positive")
    radius = int(round(4.0 * sigma))
    x = np.arange(-radius, radius + 1, dtype=np.float64)
    phi = np.exp(-0.5 / (sigma * sigma) * x ** 2)
    return phi / phi.sum()
