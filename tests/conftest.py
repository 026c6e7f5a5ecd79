import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: takes more than a few seconds")


def golden_index():
    with open(os.path.join(GOLDEN, "index.json")) as f:
        return json.load(f)


def load_golden(name):
    """Return (mask, kernel, reps, output-or-None, entry) for a golden diffusion case."""
    entry = golden_index()[name]
    z = np.load(os.path.join(GOLDEN, entry["file"]))
    if "mask" in z:
        mask = z["mask"]
    else:
        from maxibone_b200.synthetic import spheres_mask
        mask = spheres_mask(tuple(entry["shape"]), 40, (4, 20), seed=0)
    out = z["output"] if "output" in z else None
    return mask, z["kernel"], int(z["reps"]), out, entry


DIFFUSION_CASES = [k for k, v in golden_index().items() if "kernel_size" in v]
