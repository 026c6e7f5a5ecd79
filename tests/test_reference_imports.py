"""The reference's import paths resolve to this package's drop-in modules, and
the drop-in bitpacking module enforces the reference's argument rules (no GPU
needed for either)."""
import importlib
import sys

import numpy as np
import pytest

from maxibone_b200 import reference_imports

# The package re-exports the diffusion function under its own name, so take
# the modules from the import system rather than by attribute.
bp = importlib.import_module("maxibone_b200.bitpacking")
dd = importlib.import_module("maxibone_b200.diffusion")


@pytest.fixture
def clean_lib_modules():
    saved = {k: v for k, v in sys.modules.items() if k == "lib" or k.startswith("lib.")}
    yield
    for k in [k for k in sys.modules if k == "lib" or k.startswith("lib.")]:
        del sys.modules[k]
    sys.modules.update(saved)


def test_install_serves_reference_paths(clean_lib_modules):
    names = reference_imports.install()
    assert names == ["lib.cpp.gpu.diffusion", "lib.cpp.gpu.bitpacking", "lib.cpp.gpu.histograms",
                     "lib.cpp.gpu.morphology"]
    from lib.cpp.gpu.diffusion import diffusion  # noqa: E402  (the production import line)
    from lib.cpp.gpu import bitpacking  # noqa: E402
    # the histogram step's import line (src/processing_steps/1000_compute_histograms.py:20)
    from lib.cpp.gpu.histograms import axis_histograms as axis_histogram_par_gpu  # noqa: E402
    from lib.cpp.gpu.histograms import field_histogram as field_histogram_par_gpu  # noqa: E402
    hg = importlib.import_module("maxibone_b200.histograms")
    assert axis_histogram_par_gpu is hg.axis_histograms and field_histogram_par_gpu is hg.field_histogram
    import lib.cpp.gpu.morphology as lib_morphology  # noqa: E402  (src/lib/py/helpers.py:19)
    assert lib_morphology.dilate_3d_sphere_bitpacked is importlib.import_module(
        "maxibone_b200.morphology").dilate_3d_sphere_bitpacked
    assert diffusion is dd.diffusion
    assert bitpacking.encode is bp.encode and bitpacking.decode is bp.decode
    assert importlib.import_module("lib.cpp.gpu.diffusion") is dd


def test_install_cpu_paths(clean_lib_modules):
    names = reference_imports.install(cpu=True)
    assert "lib.cpp.cpu.diffusion" in names
    from lib.cpp.cpu.diffusion import diffusion  # noqa: E402
    assert diffusion is dd.diffusion


def test_bitpacking_argument_rules():
    mask = np.zeros(64, np.uint8)
    with pytest.raises(TypeError):
        bp.encode(mask.astype(bool), np.zeros(2, np.uint32))
    with pytest.raises(TypeError):
        bp.encode(mask, np.zeros(2, np.int64))
    with pytest.raises(TypeError):
        bp.decode(np.zeros(4, np.uint32)[::2], mask)
    with pytest.raises(ValueError):
        bp.encode(mask, np.zeros(1, np.uint32))
    with pytest.raises(ValueError):
        bp.encode(np.zeros(40, np.uint8), np.zeros(2, np.uint32))
