"""Batched form: many uneven device volumes in one CUDA graph (run with -m gpu).

The batched tensor-core launches do the same arithmetic per tile as the
single-volume passes, so every volume must equal its own single-volume run
exactly; FP32 batches take the per-volume CUDA-core path and must match too."""
import numpy as np
import pytest
import torch

from maxibone_b200 import device, gauss_kernel
from maxibone_b200.synthetic import spheres_mask

pytestmark = pytest.mark.gpu

SHAPES = [(96, 128, 192), (128, 96, 128), (64, 64, 64), (40, 72, 136), (33, 50, 60), (20, 30, 44), (130, 64, 256)]
SIGMAS = [2.0, 4.0, 2.0, 8.0, 2.0, 4.0, 8.0]
REPS = [3, 3, 3, 2, 3, 3, 2]


def make_batch(field):
    masks, outs, fouts, kernels = [], [], [], []
    for i, shape in enumerate(SHAPES):
        m = spheres_mask(shape, 8, (3, 9), seed=100 + i)
        masks.append(torch.from_numpy(m).cuda())
        outs.append(torch.empty(shape, dtype=torch.uint16, device="cuda"))
        fouts.append(torch.empty(shape, dtype=torch.float32, device="cuda"))
        kernels.append(gauss_kernel(SIGMAS[i]).astype(np.float32))
    return masks, outs, fouts, kernels


def single(mask, kernel, reps, field):
    out = torch.empty(mask.shape, dtype=torch.uint16, device="cuda")
    fo = torch.empty(mask.shape, dtype=torch.float32, device="cuda")
    # The batched launches run the passes the single-volume call runs by
    # default (the fused y + x kernel where it applies, else separate passes).
    device.diffuse(mask, kernel, reps, output=out, field=field, field_out=fo)
    return out, fo


@pytest.mark.parametrize("field", ["bf16", "f16", "f32"])
def test_batch_equals_single_volume_runs(field):
    masks, outs, fouts, kernels = make_batch(field)
    plan = device.BatchPlan(masks, kernels, REPS, outputs=outs, field=field, field_outs=fouts)
    text = plan.describe()
    plan.run()
    torch.cuda.synchronize()
    device.tensor_core_status()
    for i in range(len(SHAPES)):
        o, f = single(masks[i], kernels[i], REPS[i], field)
        torch.cuda.synchronize()
        assert torch.equal(outs[i], o), (i, text)
        assert torch.equal(fouts[i], f), (i, text)
    if field != "f32":
        assert "one tensor-core launch per pass" in text
    plan.close()


# Extents that are not multiples of the 128-wide tensor-core tiles leave tiles
# partly outside a volume.  32 volumes of the batched workload (dims from
# {96, ..., 512}) at 30 repetitions keep the memory system busy enough that a
# reordering of the asynchronous tile stores would show.
@pytest.mark.parametrize("field", ["bf16"])
def test_uneven_volumes_many_reps_batch_equals_single_and_repeats(field):
    from maxibone_b200.synthetic import batch_shapes, spheres_mask_torch
    reps = 30
    specs = batch_shapes(32, seed=3)
    masks = [spheres_mask_torch(sh, fg, seed=i) for i, (sh, _, fg) in enumerate(specs)]
    kernels = [gauss_kernel(sig).astype(np.float32) for _, sig, _ in specs]
    fouts = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh, _, _ in specs]
    plan = device.BatchPlan(masks, kernels, reps, field=field, field_outs=fouts)
    plan.run()
    torch.cuda.synchronize()
    device.tensor_core_status()
    plan.close()
    for i, (sh, _, _) in enumerate(specs):
        runs = []
        for _ in range(2 if i < 4 else 1):
            fo = torch.empty(sh, dtype=torch.float32, device="cuda")
            device.diffuse(masks[i], kernels[i], reps, field=field, field_out=fo)
            runs.append(fo)
        torch.cuda.synchronize()
        assert torch.equal(runs[0], runs[-1]), (i, sh)
        assert torch.equal(fouts[i], runs[0]), (i, sh)


def test_batch_with_wide_radius_volume_equals_single_runs():
    # Radius 48 is above the batched tensor-core passes' 32: that volume takes the
    # per-volume path (wide-radius tensor-core passes) inside the plan.
    from maxibone_b200.synthetic import spheres_mask
    shapes, sigmas = [(64, 96, 136), (48, 80, 128), (40, 64, 192)], [12.0, 2.0, 12.0]
    masks = [torch.from_numpy(spheres_mask(sh, 6, (3, 9), seed=40 + i)).cuda() for i, sh in enumerate(shapes)]
    kernels = [gauss_kernel(s).astype(np.float32) for s in sigmas]
    fouts = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh in shapes]
    plan = device.BatchPlan(masks, kernels, 3, field="bf16", field_outs=fouts)
    plan.run()
    torch.cuda.synchronize()
    device.tensor_core_status()
    plan.close()
    for i, sh in enumerate(shapes):
        fo = torch.empty(sh, dtype=torch.float32, device="cuda")
        device.diffuse(masks[i], kernels[i], 3, field="bf16", field_out=fo)
        torch.cuda.synchronize()
        assert torch.equal(fouts[i], fo), i


def test_batch_plan_replays():
    masks, outs, fouts, kernels = make_batch("bf16")
    plan = device.BatchPlan(masks, kernels, REPS, outputs=outs, field="bf16", field_outs=fouts)
    plan.run()
    torch.cuda.synchronize()
    first = [f.clone() for f in fouts]
    for f in fouts:
        f.zero_()
    plan.run()
    torch.cuda.synchronize()
    for a, b in zip(first, fouts):
        assert torch.equal(a, b)
    plan.close()


def test_batch_autotune_reports_and_stays_accurate():
    masks, outs, fouts, kernels = make_batch("f16")
    plan = device.BatchPlan(masks, kernels, REPS, outputs=outs, field="f16", field_outs=fouts, autotune=True)
    text = plan.describe()
    assert "tuned" in text or "cached" in text
    plan.run()
    torch.cuda.synchronize()
    for i in range(len(SHAPES)):
        want = torch.empty(SHAPES[i], dtype=torch.float64, device="cuda")
        device.diffuse(masks[i], kernels[i], REPS[i], field="f64", field_out=want)
        assert (fouts[i].double() - want).abs().max().item() < 1e-3
    plan.close()


def test_batch_autotune_persists_choices(tmp_path, monkeypatch):
    # Shapes and a radius no other test tunes, so the process has no choice for them yet.
    from maxibone_b200 import _lib
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("MAXIBONE_TUNE_CACHE", str(cache))
    shapes, sigma, reps = [(72, 80, 128), (48, 64, 192), (40, 96, 64)], 2.5, 2
    kernel = gauss_kernel(sigma).astype(np.float32)  # radius 10
    masks = [torch.from_numpy(spheres_mask(sh, 6, (3, 8), seed=7 + i)).cuda() for i, sh in enumerate(shapes)]

    def plan_and_check():
        outs = [torch.empty(sh, dtype=torch.uint16, device="cuda") for sh in shapes]
        fouts = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh in shapes]
        plan = device.BatchPlan(masks, [kernel] * 3, reps, outputs=outs, field="bf16", field_outs=fouts, autotune=True)
        text = plan.describe()
        plan.run()
        torch.cuda.synchronize()
        for m, sh, f in zip(masks, shapes, fouts):
            want = torch.empty(sh, dtype=torch.float64, device="cuda")
            device.diffuse(m, kernel, reps, field="f64", field_out=want)
            assert (f.double() - want).abs().max().item() <= 2e-3
        plan.close()
        return text

    _lib.check(_lib.lib().maxi_batch_tune_forget())
    first = plan_and_check()
    assert "tuned: batched" in first and "per_volume_tc" in first and "cuda_cores" in first, first
    text = cache.read_text()
    gpu = torch.cuda.get_device_name()
    key = f"{gpu} sm{torch.cuda.get_device_properties(0).multi_processor_count}|bf16|r10|"
    lines = [ln for ln in text.splitlines() if key in ln]
    assert len(lines) == 1 and '"form": ' in lines[0] and "40x96x64,48x64x192,72x80x128" in lines[0], text
    assert "cached choice" in plan_and_check()
    # A choice read from the file (here forced to the CUDA-core passes) is used
    # without timing, after the process forgets its own.
    forced = lines[0].split('"form": ')[0] + '"form": "cuda_cores"}'
    cache.write_text('{\n"entries": {\n' + forced + "\n}\n}\n")
    _lib.check(_lib.lib().maxi_batch_tune_forget())
    text = plan_and_check()
    assert "cached choice" in text and "-> cuda_cores" in text and "per-volume CUDA-core passes" in text, text
    _lib.check(_lib.lib().maxi_batch_tune_forget())


def test_batch_rejects_bad_volumes():
    m = torch.zeros((4, 4, 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(ValueError):
        device.BatchPlan([m], [np.ones(4, np.float32)], 1, outputs=[torch.empty((4, 4, 4), dtype=torch.uint16, device="cuda")])
    with pytest.raises(ValueError):
        device.BatchPlan([m], [gauss_kernel(1)], 1, outputs=None)
