"""C ABI checks that need no GPU: the library loads, exports every function
include/*.h declares, and rejects malformed arguments before touching a device."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from maxibone_b200 import _lib


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(maxi_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    names = declared_functions()
    assert "maxi_diffusion_in_memory" in names
    for name in names:
        assert hasattr(lib, name), f"{name} declared in include/ but not exported"
    assert set(names) <= set(_lib.SIGNATURES), "ctypes signatures missing for some declared symbols"


def declared_parameter_counts():
    """{function: number of parameters} from the prototypes in include/*.h."""
    counts = {}
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"\b(maxi_[a-z0-9_]+)\s*\(([^;{]*?)\)\s*;", text):
            params = m.group(2).strip()
            counts[m.group(1)] = 0 if params in ("", "void") else params.count(",") + 1
    return counts


def test_ctypes_signatures_match_the_header_prototypes():
    counts = declared_parameter_counts()
    assert len(counts) == len(declared_functions())
    for name, n in counts.items():
        restype, argtypes = _lib.SIGNATURES[name]
        assert len(argtypes) == n, f"{name}: header has {n} parameters, ctypes binding {len(argtypes)}"
        if name == "maxi_diffusion_workspace_size":
            assert restype is ctypes.c_int64
        elif name in ("maxi_last_error", "maxi_version"):
            assert restype is ctypes.c_char_p
        else:
            assert restype is ctypes.c_int, name


def test_version_string():
    assert b"sm_100a" in _lib.lib().maxi_version()


def _call_in_memory(mask, kernel, out, reps=1):
    nz, ny, nx = mask.shape if mask is not None else (1, 1, 1)
    return _lib.lib().maxi_diffusion_in_memory(
        mask.ctypes.data if mask is not None else None, nz, ny, nx,
        kernel.ctypes.data if kernel is not None else None, kernel.shape[0] if kernel is not None else 0,
        reps, out.ctypes.data if out is not None else None, 0)


def test_invalid_arguments_are_reported_before_device_use():
    m = np.zeros((4, 4, 4), np.uint8)
    k = np.ones(3, np.float32) / 3
    o = np.zeros((4, 4, 4), np.uint16)
    lib = _lib.lib()
    assert _call_in_memory(None, k, o) == 1
    assert b"mask" in lib.maxi_last_error()
    assert _call_in_memory(m, None, o) == 1
    assert _call_in_memory(m, k, None) == 1
    assert _call_in_memory(m, np.ones(4, np.float32), o) == 1  # even length
    assert b"odd" in lib.maxi_last_error()
    assert _call_in_memory(m, k, o, reps=-1) == 1
    assert lib.maxi_diffusion_in_memory(m.ctypes.data, 0, 4, 4, k.ctypes.data, 3, 1, o.ctypes.data, 0) == 1
    big = np.ones(2 * 1025 + 1, np.float32)
    assert _call_in_memory(m, big, o) == 5  # radius above the supported maximum


def test_device_entry_rejects_bad_enums():
    lib = _lib.lib()
    k = np.ones(3, np.float32) / 3
    dummy = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    assert lib.maxi_diffusion_device(dummy, 7, 4, 4, 4, k.ctypes.data, 3, 1, dummy, None, 0, 0, None, 0, None) == 1
    assert lib.maxi_diffusion_device(dummy, 0, 4, 4, 4, k.ctypes.data, 3, 1, dummy, None, 9, 0, None, 0, None) == 1
    # reference rounding is FP32-only
    assert lib.maxi_diffusion_device(dummy, 0, 4, 4, 4, k.ctypes.data, 3, 1, dummy, None, 1, 1, None, 0, None) == 1
    assert lib.maxi_diffusion_device(dummy, 0, 4, 4, 4, k.ctypes.data, 3, 1, None, None, 0, 0, None, 0, None) == 1


def test_workspace_size():
    lib = _lib.lib()
    # two field buffers (256-byte rounded) + the bit-packed mask (32 words -> 256 bytes)
    assert lib.maxi_diffusion_workspace_size(10, 10, 10, 0) == 2 * 4096 + 256
    assert lib.maxi_diffusion_workspace_size(10, 10, 10, 1) == 2 * 2048 + 256
    assert lib.maxi_diffusion_workspace_size(0, 10, 10, 0) == -1
    assert lib.maxi_diffusion_workspace_size(10, 10, 10, 42) == -1


def test_bitpack_rejects_bad_sizes():
    lib = _lib.lib()
    dummy = ctypes.c_void_p(16)
    assert lib.maxi_bitpack_encode(dummy, 33, dummy, None) == 1
    assert lib.maxi_bitpack_decode(None, 32, dummy, None) == 1


def test_no_device_is_an_error_not_a_fallback():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is visible")
    m = np.zeros((4, 4, 4), np.uint8)
    k = np.ones(3, np.float32) / 3
    o = np.zeros((4, 4, 4), np.uint16)
    assert _call_in_memory(m, k, o) == 6


def test_device_entry_rejects_misaligned_workspace_and_packed_mask():
    # Both are rejected on the host, before any device work: the passes read the
    # workspace with 16-byte vector / TMA loads and a bit-packed mask as words.
    lib = _lib.lib()
    k = np.ones(3, np.float32) / 3
    mask, out = ctypes.c_void_p(4096), ctypes.c_void_p(8192)  # never dereferenced
    ws_bytes = lib.maxi_diffusion_workspace_size(4, 4, 32, 0)
    for off in (1, 16, 128):
        rc = lib.maxi_diffusion_device(mask, 0, 4, 4, 32, k.ctypes.data, 3, 1, out, None, 0, 0,
                                       ctypes.c_void_p(65536 + off), ws_bytes, None)
        assert rc == 1 and b"256-byte" in lib.maxi_last_error()
    rc = lib.maxi_diffusion_device(ctypes.c_void_p(4098), 1, 4, 4, 32, k.ctypes.data, 3, 1, out, None, 0, 0,
                                   None, 0, None)
    assert rc == 1 and b"4-byte" in lib.maxi_last_error()
    rc = lib.maxi_diffusion_device_noalloc(ctypes.c_void_p(4098), 1, 4, 4, 32, k.ctypes.data, 3, 1, out, None, None)
    assert rc == 1 and b"4-byte" in lib.maxi_last_error()


def test_keep_device_buffers_and_last_path_need_no_device():
    lib = _lib.lib()
    assert lib.maxi_keep_device_buffers(1) == 0
    assert lib.maxi_keep_device_buffers(0) == 0
    assert lib.maxi_last_path() >= 0
