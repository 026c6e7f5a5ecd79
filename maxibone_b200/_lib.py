"""ctypes binding of the in-tree CUDA library ``libmaxibone_diffusion.so``.

The library is the product: every diffusion call goes through it.  If it is
missing the import fails loudly (there is no CPU fallback); build it with
``python -m maxibone_b200.build`` or ``__graft_entry__.build()``.
"""
from __future__ import annotations

import ctypes
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libmaxibone_diffusion.so")

MAXI_OK = 0
STATUS_NAMES = {
    0: "MAXI_OK", 1: "MAXI_ERR_INVALID_ARGUMENT", 2: "MAXI_ERR_CUDA", 3: "MAXI_ERR_OUT_OF_MEMORY",
    4: "MAXI_ERR_IO", 5: "MAXI_ERR_UNSUPPORTED", 6: "MAXI_ERR_NO_DEVICE",
}
FIELD_TYPES = {"f32": 0, "bf16": 1, "f16": 2, "f64": 3}
MASK_FORMATS = {"u8": 0, "bitpacked": 1}
FLAG_REFERENCE_ROUNDING = 0x1
FLAG_NO_TENSOR_CORES = 0x2
FLAG_NEAREST_ROUNDING = 0x4
FLAG_MASK_FROM_FIELD = 0x8
FLAG_AUTOTUNE = 0x10
FLAG_SEPARATE_PASSES = 0x20
FLAG_SPLIT_COEFFICIENTS = 0x40
PATH_CUDA_CORES = 0x1
PATH_TENSOR_CORES_ZY = 0x2
PATH_TENSOR_CORES_X = 0x4
PATH_FUSED_YX = 0x8
PATH_GENERIC = 0x10
PATH_FP32_FALLBACK = 0x20


class MaxiVolume(ctypes.Structure):
    """The C struct maxi_volume."""
    _fields_ = [("mask", ctypes.c_void_p), ("output", ctypes.c_void_p), ("field_out", ctypes.c_void_p),
                ("nz", ctypes.c_int64), ("ny", ctypes.c_int64), ("nx", ctypes.c_int64),
                ("kernel", ctypes.c_void_p), ("kernel_size", ctypes.c_int64), ("repititions", ctypes.c_int64)]

# Every symbol include/maxibone_diffusion.h declares, with (restype, argtypes).
_i64, _i32, _p, _int = ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_int
SIGNATURES = {
    "maxi_last_error": (ctypes.c_char_p, []),
    "maxi_version": (ctypes.c_char_p, []),
    "maxi_diffusion_in_memory": (_int, [_p, _i64, _i64, _i64, _p, _i64, _i64, _p, _int]),
    "maxi_diffusion_workspace_size": (_i64, [_i64, _i64, _i64, _i32]),
    "maxi_diffusion_device": (_int, [_p, _i32, _i64, _i64, _i64, _p, _i64, _i64, _p, _p, _i32, _i32, _p, _i64, _p]),
    "maxi_diffusion_device_ex": (_int, [_p, _i32, _i64, _i64, _i64, _p, _i64, _i64, _p, _p, _i32, _i32, _p, _i64,
                                        _p, _p, _i64, _i64]),
    "maxi_bitpack_encode": (_int, [_p, _i64, _p, _p]),
    "maxi_bitpack_decode": (_int, [_p, _i64, _p, _p]),
    "maxi_combine_fields": (_int, [_p, _p, _i64, _i64, _i64, _p, _p]),
    "maxi_mask_cylinder": (_int, [_p, _i64, _i64, _i64, _p]),
    "maxi_morphology_sphere": (_int, [_p, _p, _i64, _i64, _i64, _i64, _int, _p]),
    "maxi_morphology_sphere_bitpacked": (_int, [_p, _p, _i64, _i64, _i64, _i64, _int, _p]),
    "maxi_implant_masks": (_int, [_p, _i64, _i64, _i64, ctypes.c_float, _p, _p, _p, _p, _p, _p, _p, _p, _p]),
    "maxi_field_histogram": (_int, [_p, _i64, _i64, _i64, _p, _i64, _i64, _i64, _i64, _i64, _p, _i64, _i64,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, _p]),
    "maxi_axis_histograms": (_int, [_p, _i64, _i64, _i64, _i64, _i64, _i64, _i64, _p, _p, _p, _p, _i64, _i64,
                                    _i64, _i64, ctypes.c_double, ctypes.c_double, _p]),
    "maxi_diffusion_device_noalloc": (_int, [_p, _i32, _i64, _i64, _i64, _p, _i64, _i64, _p, _p, _p]),
    "maxi_tensor_core_status": (_int, []),
    "maxi_tensor_core_taps": (_int, [_p, _i64, _i32, _p, _p]),
    "maxi_release_cached_memory": (_int, []),
    "maxi_keep_device_buffers": (_int, [_int]),
    "maxi_last_path": (_int, []),
    "maxi_batch_plan_create": (_int, [_p, _i64, _i32, _i32, _p, ctypes.POINTER(ctypes.c_void_p)]),
    "maxi_batch_plan_run": (_int, [_p, _p]),
    "maxi_batch_plan_describe": (_int, [_p, ctypes.c_char_p, _i64]),
    "maxi_batch_plan_destroy": (_int, [_p]),
    "maxi_batch_tune_forget": (_int, []),
    "maxi_diffusion_batched": (_int, [_p, _i64, _i32, _i32, _p]),
    "maxi_diffusion_out_of_core": (_int, [_p, _i64, _i64, _i64, _i64, _i64, _i64, _p, _i64, _i64, _p, _int]),
    "maxi_diffusion_out_of_core_ex": (_int, [_p, _i64, _i64, _i64, _i64, _p, _i64, _i64, _p, _i32, _i32, _int]),
    "maxi_diffusion_on_disk": (_int, [ctypes.c_char_p, _p, _i64, ctypes.c_char_p, _i64, _i64, _i64, _i64, _i64,
                                      _i64, _i64, _int]),
    "maxi_out_of_core_plan": (_int, [_i64, _i64, _i64, _i64, _i64, _i64, _i32, _i32, _i64, _p, _p, _p]),
    "maxi_profile_enable": (_int, [_int]),
    "maxi_profile_read": (_int, [_p, _p, _i32]),
}
KERNEL_KINDS = ["init", "z", "y", "x", "x_final", "yx", "other", "spare"]


class MaxiError(RuntimeError):
    """A nonzero maxi_status, with the library's message."""

    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {message}")
        self.code = code


_LIB = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run `python -m maxibone_b200.build`")
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = handle
    return _LIB


def check(code: int) -> None:
    if code != MAXI_OK:
        msg = lib().maxi_last_error()
        msg = msg.decode() if msg else ""
        if code == 1:
            raise ValueError(f"{STATUS_NAMES[code]}: {msg}")
        if code == 3:
            raise MemoryError(f"{STATUS_NAMES[code]}: {msg}")
        raise MaxiError(code, msg)
