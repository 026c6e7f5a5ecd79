"""maxibone_b200: maxibone's 3-D mask-diffusion path on NVIDIA B200 (sm_100a).

The product is the CUDA library ``libmaxibone_diffusion.so`` (C ABI in
include/maxibone_diffusion.h).  This package holds its Python side:

* ``maxibone_b200.diffusion.diffusion``: drop-in for the reference pybind
  module ``diffusion`` (both overloads, same argument names and defaults).
* ``maxibone_b200.device``: the same path on torch CUDA tensors (device
  resident, stream ordered, reduced-precision field forms, bit-packed masks).
* ``maxibone_b200.kernels.gauss_kernel``: the reference's kernel builder.
"""
from .kernels import gauss_kernel  # noqa: F401
from .diffusion import diffusion  # noqa: F401

__all__ = ["diffusion", "gauss_kernel"]
