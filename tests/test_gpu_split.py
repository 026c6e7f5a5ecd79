"""The z-slab split of one volume (maxibone_b200.zsplit) with the library's
CUDA slab step, on one GPU (run with -m gpu): the slabs run one after another
in one process and exchange halos by device copies, so no kernel waits on
another.  This is the split the ranks of a multi-GPU run perform, with the
same slab rounds (maxi_diffusion_device_ex: start from the slab's field,
shrinking plane windows on cut sides).  FP32 results equal the single-volume
call bit for bit; the 16-bit forms stay within their bounds of the FP64 form."""
import numpy as np
import pytest
import torch

from maxibone_b200 import device, gauss_kernel
from maxibone_b200.synthetic import spheres_mask
from maxibone_b200.zsplit import diffuse_slabs_in_process, library_step, split_plan

pytestmark = pytest.mark.gpu


def _whole(mask, kernel, reps, field):
    out = torch.empty(mask.shape, dtype=torch.uint16, device="cuda")
    fo = torch.empty(mask.shape, dtype=torch.float64 if field == "f64" else torch.float32, device="cuda")
    device.diffuse(mask, kernel, reps, output=out, field=field, field_out=fo)
    torch.cuda.synchronize()
    return out, fo


@pytest.mark.parametrize("shape,sigma,reps,world,k", [((70, 64, 96), 2.0, 9, 3, None), ((40, 30, 45), 1.0, 6, 2, 2),
                                                      ((96, 40, 128), 2.0, 7, 4, 1), ((33, 20, 64), 1.5, 5, 1, None)])
def test_split_fp32_equals_single_volume(shape, sigma, reps, world, k):
    mask = torch.from_numpy(spheres_mask(shape, 10, (2, 8), seed=sum(shape))).cuda()
    kernel = gauss_kernel(sigma).astype(np.float32)
    plan = split_plan(shape[0], world, kernel.shape[0] // 2, reps, k)
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    fo = torch.empty(shape, dtype=torch.float32, device="cuda")
    diffuse_slabs_in_process(mask, kernel, plan, library_step("f32"), output=out, field_out=fo)
    torch.cuda.synchronize()
    want_u16, want = _whole(mask, kernel, reps, "f32")
    assert plan.rounds > 1 or world == 1
    assert torch.equal(fo, want)
    assert torch.equal(out, want_u16)


@pytest.mark.parametrize("field", ["bf16", "f16"])
def test_split_16bit_within_bounds(field):
    shape, reps = (64, 128, 256), 12
    mask = torch.from_numpy(spheres_mask(shape, 20, (3, 12), seed=5)).cuda()
    kernel = gauss_kernel(3.0).astype(np.float32)  # radius 12
    plan = split_plan(shape[0], 2, kernel.shape[0] // 2, reps)
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    fo = torch.empty(shape, dtype=torch.float32, device="cuda")
    diffuse_slabs_in_process(mask, kernel, plan, library_step(field), output=out, field_out=fo)
    torch.cuda.synchronize()
    device.tensor_core_status()
    _, want = _whole(mask, kernel, reps, "f64")
    assert plan.rounds > 1
    assert float((fo.double() - want).abs().max()) <= {"bf16": 2e-3, "f16": 5e-4}[field]
    assert bool((out.view(torch.int16)[mask > 0] == -1).all())
