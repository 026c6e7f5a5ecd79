"""Field steps after the diffusion in maxibone's pipeline.

``combine_fields(gauss_field, edt_field)`` is the Gaussian + EDT combination of
src/processing_steps/0975_combine_fields.py:38-62 -- the normalised difference
of the two uint16 fields, shifted and rescaled, masked by the implant cylinder
and converted to uint16 with the reference's to_int (normalized_convert,
src/lib/cpp/include/general.hh:78-118) -- bit-identical to the script, on the
GPU.  A maintainer replaces the script's numpy block (from ``edt_max = ...`` to
the second ``combined *= cylinder_mask``) with

    combined = combine_fields(gauss_field, edt_field)

Both fields are uint16 [nz, ny, nx] numpy arrays (as the pipeline saves them)
or CUDA tensors; the cylinder spans y and x as generate_cylinder_mask(ny, nx),
which is the script's generate_cylinder_mask(nx) for its square planes.

``mask_cylinder(field)`` is the diffusion step's ``result * cylinder_mask``
before it saves the field (src/processing_steps/0900_generate_gauss_c.py:117,124):
the voxels outside the implant cylinder become 0.
"""
from __future__ import annotations

import numpy as np

from . import _lib


def combine_fields(gauss_field, edt_field, output=None):
    """uint16 combination of the two fields (numpy arrays in, numpy array out;
    or uint16/int16 CUDA tensors in, tensor out, stream-ordered on the current
    stream and synchronised)."""
    import torch

    on_device = isinstance(gauss_field, torch.Tensor)
    if on_device:
        g, e = gauss_field, edt_field
        if not (g.is_cuda and e.is_cuda):
            raise ValueError("tensor fields must be CUDA tensors")
        if g.dtype not in (torch.uint16, torch.int16) or e.dtype not in (torch.uint16, torch.int16):
            raise TypeError("fields must be uint16 (or int16 holding uint16 bits)")
        g, e = g.contiguous(), e.contiguous()
    else:
        ga, ea = np.asarray(gauss_field), np.asarray(edt_field)
        if ga.dtype != np.uint16 or ea.dtype != np.uint16:
            raise TypeError("fields must be uint16 arrays")
        g = torch.from_numpy(np.ascontiguousarray(ga).view(np.int16)).cuda()
        e = torch.from_numpy(np.ascontiguousarray(ea).view(np.int16)).cuda()
    if g.dim() != 3 or tuple(g.shape) != tuple(e.shape):
        raise ValueError(f"fields must be 3-D and of one shape, got {tuple(g.shape)} and {tuple(e.shape)}")
    nz, ny, nx = g.shape
    out = output if (on_device and output is not None) else torch.empty(g.shape, dtype=g.dtype, device=g.device)
    st = torch.cuda.current_stream()
    _lib.check(_lib.lib().maxi_combine_fields(g.data_ptr(), e.data_ptr(), nz, ny, nx, out.data_ptr(),
                                              st.cuda_stream))
    if on_device:
        return out
    return out.cpu().numpy().view(np.uint16)


def mask_cylinder(field):
    """field * generate_cylinder_mask(ny, nx): a new uint16 numpy array for a numpy
    field, or the uint16/int16 CUDA tensor itself, masked in place."""
    import torch

    if isinstance(field, torch.Tensor):
        if not field.is_cuda or field.dtype not in (torch.uint16, torch.int16) or not field.is_contiguous():
            raise TypeError("field must be a contiguous uint16 (or int16) CUDA tensor")
        t = field
    else:
        a = np.asarray(field)
        if a.dtype != np.uint16:
            raise TypeError("field must be a uint16 array")
        t = torch.from_numpy(np.ascontiguousarray(a).view(np.int16)).cuda()
    if t.dim() != 3:
        raise ValueError(f"field must be 3-D, got {tuple(t.shape)}")
    nz, ny, nx = t.shape
    _lib.check(_lib.lib().maxi_mask_cylinder(t.data_ptr(), nz, ny, nx, torch.cuda.current_stream().cuda_stream))
    if isinstance(field, torch.Tensor):
        return field
    return t.cpu().numpy().view(np.uint16)
