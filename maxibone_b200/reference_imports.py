"""Serve the reference's import paths from this package.

maxibone's processing steps import the diffusion path as
``from lib.cpp.gpu.diffusion import diffusion`` (src/processing_steps/
0900_generate_gauss_c.py:17, src/test/test_diffusion.py:17) and the mask
packing as ``lib.cpp.gpu.bitpacking`` (src/lib/py/helpers.py); the histogram
step imports ``axis_histograms`` and ``field_histogram`` from
``lib.cpp.gpu.histograms`` (src/processing_steps/1000_compute_histograms.py:20), and
the mask preparation reaches the sphere morphology as ``lib.cpp.gpu.morphology``
(src/lib/py/helpers.py:19).
``install()``
registers this package's drop-in modules under those dotted names, so that
such code runs unchanged on the B200 library:

    import maxibone_b200.reference_imports as ri
    ri.install()                      # lib.cpp.gpu.{diffusion, bitpacking, histograms, morphology}
    from lib.cpp.gpu.diffusion import diffusion

``install(cpu=True)`` also routes ``lib.cpp.cpu.*`` (the OpenMP build's import
path) here.  Parent packages that already import (a real ``lib`` tree on the
path) are kept; only the leaf modules are replaced.
"""
from __future__ import annotations

import importlib
import sys
import types

_LEAVES = {"diffusion": "maxibone_b200.diffusion", "bitpacking": "maxibone_b200.bitpacking",
           "histograms": "maxibone_b200.histograms", "morphology": "maxibone_b200.morphology"}


def _package(name: str) -> types.ModuleType:
    mod = sys.modules.get(name)
    if mod is None:
        try:
            mod = importlib.import_module(name)
        except ImportError:
            mod = types.ModuleType(name)
            mod.__path__ = []  # a namespace for the leaves below
            sys.modules[name] = mod
    return mod


def install(cpu: bool = False) -> list[str]:
    """Registers lib.cpp.gpu.diffusion / .bitpacking / .histograms / .morphology (and lib.cpp.cpu.* with
    cpu=True); returns the module names it registered."""
    done = []
    for backend in ("gpu", "cpu") if cpu else ("gpu",):
        parent = None
        for name in ("lib", "lib.cpp", f"lib.cpp.{backend}"):
            pkg = _package(name)
            if parent is not None:
                setattr(parent, name.rsplit(".", 1)[1], pkg)
            parent = pkg
        for leaf, target in _LEAVES.items():
            mod = importlib.import_module(target)
            full = f"lib.cpp.{backend}.{leaf}"
            sys.modules[full] = mod
            setattr(parent, leaf, mod)
            done.append(full)
    return done
