"""Device-resident API: the diffusion on torch CUDA tensors, enqueued on the
current torch stream (torch supplies device memory and streams; the work is
the library's CUDA kernels).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib

_FIELD_OUT_DTYPE = {"f32": torch.float32, "bf16": torch.float32, "f16": torch.float32, "f64": torch.float64}


def workspace_bytes(shape, field: str = "f32") -> int:
    nz, ny, nx = shape
    n = _lib.lib().maxi_diffusion_workspace_size(nz, ny, nx, _lib.FIELD_TYPES[field])
    if n < 0:
        raise ValueError(f"invalid shape {shape} or field type {field}")
    return int(n)


def diffuse(mask: torch.Tensor, kernel, repititions: int, output: torch.Tensor | None = None,
            field: str = "f32", field_out: torch.Tensor | None = None, shape=None,
            reference_rounding: bool = False, workspace: torch.Tensor | None = None,
            stream: torch.cuda.Stream | None = None, tensor_cores: bool = True,
            error_feedback: bool = True, fuse_passes: bool = True, split_coefficients: bool = False) -> None:
    """Run the diffusion on device buffers.

    mask: uint8 [nz, ny, nx] CUDA tensor (set when > 0), or a bit-packed int32/uint32
          tensor of ceil(N/32) words (MSB first) together with `shape`.
    kernel: 1-D array-like of odd length (host values; cast to float32).
    output: uint16 CUDA tensor of the volume's shape, or None.
    field: storage type between passes: "f32", "bf16", "f16" or "f64".
    field_out: final field before quantisation (float32; float64 for "f64"), or None.
    workspace: uint8 CUDA tensor of at least workspace_bytes(shape, field), or None.
    tensor_cores: 16-bit fields: z and y passes on tcgen05 tensor cores where supported.
    error_feedback: 16-bit fields: error-feedback rounding along x (else round to nearest).
    fuse_passes: 16-bit tensor-core fields, radius 4 to 32: the y and x passes in one
          kernel per z-plane tile (else two kernels, two HBM round trips).
    split_coefficients: 16-bit tensor-core passes: high + low 16-bit coefficient halves
          (two MMAs per K step, separate y and x passes) instead of one set whose
          taps keep the kernel's sum and second moment (the default from radius 4;
          smaller radii always use the halves).
    """
    if not mask.is_cuda:
        raise ValueError("mask must be a CUDA tensor")
    if mask.dtype == torch.uint8:
        if mask.dim() != 3:
            raise ValueError(f"uint8 mask must be 3-D, got {tuple(mask.shape)}")
        fmt, (nz, ny, nx) = _lib.MASK_FORMATS["u8"], mask.shape
    elif mask.dtype in (torch.int32, torch.uint32):
        if shape is None:
            raise ValueError("a bit-packed mask needs `shape`")
        nz, ny, nx = shape
        if mask.numel() < (nz * ny * nx + 31) // 32:
            raise ValueError("bit-packed mask has too few words for the shape")
        fmt = _lib.MASK_FORMATS["bitpacked"]
    else:
        raise ValueError(f"unsupported mask dtype {mask.dtype}")
    if not mask.is_contiguous():
        raise ValueError("mask must be contiguous")
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    if k.ndim != 1:
        raise ValueError("kernel must be 1-D")
    n = nz * ny * nx
    if output is not None:
        if output.dtype != torch.uint16 or not output.is_cuda or not output.is_contiguous() or output.numel() != n:
            raise ValueError("output must be a contiguous CUDA uint16 tensor with one element per voxel")
    if field_out is not None:
        want = _FIELD_OUT_DTYPE[field]
        if field_out.dtype != want or not field_out.is_cuda or not field_out.is_contiguous() or field_out.numel() != n:
            raise ValueError(f"field_out must be a contiguous CUDA {want} tensor with one element per voxel")
    ws_ptr, ws_bytes = None, 0
    if workspace is not None:
        ws_ptr, ws_bytes = workspace.data_ptr(), workspace.numel() * workspace.element_size()
    st = stream if stream is not None else torch.cuda.current_stream(mask.device)
    flags = _lib.FLAG_REFERENCE_ROUNDING if reference_rounding else 0
    if not tensor_cores:
        flags |= _lib.FLAG_NO_TENSOR_CORES
    if not error_feedback:
        flags |= _lib.FLAG_NEAREST_ROUNDING
    if not fuse_passes:
        flags |= _lib.FLAG_SEPARATE_PASSES
    if split_coefficients:
        flags |= _lib.FLAG_SPLIT_COEFFICIENTS
    with torch.cuda.device(mask.device):
        _lib.check(_lib.lib().maxi_diffusion_device(
            mask.data_ptr(), fmt, nz, ny, nx, k.ctypes.data, k.shape[0], int(repititions),
            output.data_ptr() if output is not None else None,
            field_out.data_ptr() if field_out is not None else None,
            _lib.FIELD_TYPES[field], flags, ws_ptr, ws_bytes, st.cuda_stream))


def last_path() -> int:
    """MAXI_PATH_* bits of the kernels the last diffuse() call on this thread
    enqueued (e.g. _lib.PATH_TENSOR_CORES_ZY | _lib.PATH_TENSOR_CORES_X)."""
    return int(_lib.lib().maxi_last_path())


def bitpack(mask: torch.Tensor, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """uint8 CUDA mask -> int32 words (uint32 bit patterns), MSB first, `mask & 1`
    per voxel (the reference bitpacking.encode).  The mask is padded with zeros
    to a multiple of 32 voxels."""
    flat = mask.reshape(-1)
    n = flat.numel()
    if n % 32:
        flat = torch.cat([flat, flat.new_zeros(32 - n % 32)])
    out = torch.empty(flat.numel() // 32, dtype=torch.int32, device=mask.device)
    st = stream if stream is not None else torch.cuda.current_stream(mask.device)
    with torch.cuda.device(mask.device):
        _lib.check(_lib.lib().maxi_bitpack_encode(flat.data_ptr(), flat.numel(), out.data_ptr(), st.cuda_stream))
    return out


def bitunpack(packed: torch.Tensor, n: int, stream: torch.cuda.Stream | None = None) -> torch.Tensor:
    """int32/uint32 words -> uint8 {0,1} per voxel (the reference bitpacking.decode)."""
    n32 = (n + 31) // 32 * 32
    out = torch.empty(n32, dtype=torch.uint8, device=packed.device)
    st = stream if stream is not None else torch.cuda.current_stream(packed.device)
    with torch.cuda.device(packed.device):
        _lib.check(_lib.lib().maxi_bitpack_decode(packed.data_ptr(), n32, out.data_ptr(), st.cuda_stream))
    return out[:n]


def profile_enable(on: bool = True) -> None:
    """Bracket every library kernel launch with CUDA events (see maxi_profile_read)."""
    _lib.check(_lib.lib().maxi_profile_enable(1 if on else 0))


def profile_read() -> dict:
    """{kind: (total device ms, launches)} since the last read; waits for the events."""
    import ctypes
    n = len(_lib.KERNEL_KINDS)
    ms = (ctypes.c_double * n)()
    cnt = (ctypes.c_int64 * n)()
    _lib.check(_lib.lib().maxi_profile_read(ctypes.addressof(ms), ctypes.addressof(cnt), n))
    return {k: (ms[i], cnt[i]) for i, k in enumerate(_lib.KERNEL_KINDS) if cnt[i]}


def tensor_core_status() -> None:
    """Raise if a tensor-core pass gave up on a bounded wait since the last check."""
    _lib.check(_lib.lib().maxi_tensor_core_status())


class BatchPlan:
    """Many device volumes, each with its own kernel and repetition count, run
    as one CUDA graph (see maxi_batch_plan_create).  Build once, run many times.

    masks / outputs: lists of uint8 / uint16 CUDA tensors; field_outs: optional
    list of float32 tensors (or None entries); kernels: one 1-D array per volume
    (or one for all); reps: an int or one per volume."""

    def __init__(self, masks, kernels, reps, outputs=None, field="bf16", field_outs=None, autotune=False,
                 tensor_cores=True, error_feedback=True, stream=None, split_coefficients=False):
        import ctypes
        n = len(masks)
        if not isinstance(kernels, (list, tuple)):
            kernels = [kernels] * n
        if isinstance(reps, int):
            reps = [reps] * n
        outputs = outputs if outputs is not None else [None] * n
        field_outs = field_outs if field_outs is not None else [None] * n
        self._keep = [np.ascontiguousarray(k, dtype=np.float32) for k in kernels]
        self._tensors = (list(masks), list(outputs), list(field_outs))
        arr = (_lib.MaxiVolume * n)()
        for i in range(n):
            m, o, f = masks[i], outputs[i], field_outs[i]
            if m.dtype != torch.uint8 or not m.is_cuda or not m.is_contiguous() or m.dim() != 3:
                raise ValueError("masks must be contiguous 3-D uint8 CUDA tensors")
            for t, dt in ((o, torch.uint16), (f, torch.float32)):
                if t is not None and (t.dtype != dt or not t.is_cuda or not t.is_contiguous() or t.shape != m.shape):
                    raise ValueError(f"outputs must be contiguous {dt} CUDA tensors shaped like their masks")
            nz, ny, nx = m.shape
            k = self._keep[i]
            arr[i] = _lib.MaxiVolume(m.data_ptr(), o.data_ptr() if o is not None else None,
                                     f.data_ptr() if f is not None else None, nz, ny, nx, k.ctypes.data, k.shape[0],
                                     int(reps[i]))
        flags = (_lib.FLAG_AUTOTUNE if autotune else 0) | (0 if tensor_cores else _lib.FLAG_NO_TENSOR_CORES) | \
            (0 if error_feedback else _lib.FLAG_NEAREST_ROUNDING) | \
            (_lib.FLAG_SPLIT_COEFFICIENTS if split_coefficients else 0)
        st = stream if stream is not None else torch.cuda.current_stream()
        self._plan = ctypes.c_void_p()
        _lib.check(_lib.lib().maxi_batch_plan_create(ctypes.addressof(arr), n, _lib.FIELD_TYPES[field], flags,
                                                     st.cuda_stream, ctypes.byref(self._plan)))

    def run(self, stream=None):
        st = stream if stream is not None else torch.cuda.current_stream()
        _lib.check(_lib.lib().maxi_batch_plan_run(self._plan, st.cuda_stream))

    def describe(self) -> str:
        import ctypes
        buf = ctypes.create_string_buffer(1 << 14)
        _lib.check(_lib.lib().maxi_batch_plan_describe(self._plan, buf, len(buf)))
        return buf.value.decode()

    def close(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value and _lib is not None:
            _lib.lib().maxi_batch_plan_destroy(plan)
        self._plan = None

    def __del__(self):
        self.close()
