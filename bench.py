#!/usr/bin/env python
"""Throughput benchmark of the mask-diffusion path on B200.

Headline workload (`value`): a 1024^3 uint8 mask shaped like a bone sample with
a metal implant (solid cylinder of radius 120 voxels along z through the centre
plus seeded value-noise structures, ~25% foreground), a normalised Gaussian
with sigma = 8 (radius 32, 65 taps, float32), R = 100 repetitions, FP32 field,
uint16 output.  One step = one full diffusion call over the resident mask
(mask -> field, 100 x (z, y, x, re-illuminate), quantise).

Metric: Gvox*rep/s = voxels * repetitions * steps / device time (whole job,
summed over ranks).  Each rank diffuses its own volume (independent units, no
collective): scaling is weak.

Also reported on the same line:
  roofline      the repetition's algorithmic HBM bytes, V R (2 s_field + s_mask)
                (9 B per voxel-repetition for the FP32 field with a uint8 mask,
                4.125 B for a 16-bit field with the bit-packed mask), over the
                device time, against the measured HBM copy bandwidth; the
                dominant kernel's own figure beside it;
  e2e           the same metric through the reference-facing host call, numpy
                in and out, from pinned and from pageable host buffers;
  cfg0          the 128^3 sphere mask, sigma 3, R = 10, FP32, beside the
                reference module on the same input;
  precision     the 1024^3 mask bit-packed, BF16 and FP16 fields (the z, y and x
                tensor-core passes; the fused y + x kernel; the split coefficient
                halves; CUDA cores), R = 100 and R = 500, max / mean abs error
                against the FP64 form and the FP32 form; sigma = 32 (257 taps),
                CUDA-core stencil vs banded-Toeplitz tensor cores;
  batched       64 uneven volumes, sigma in {2, 4, 8}, R = 50, BF16 plan vs
                per-volume FP32 launches, error of every volume vs FP64;
  out_of_core   3456 x 3456 x 4096 (z, y, x) mask streamed from pinned host
                memory, sigma 8, R = 20, BF16, end to end (PCIe included);
  cpu_baseline  the reference's OpenMP CPU module (oracle/_ref, built from the
                reference sources) timed on this host on a bounded sample;
  fields, morphology, implant_masks   the steps either side of the path,
                beside the reference's own CPU modules on bounded samples.
Each section carries the SM clocks sampled while it ran.

`--impl reference` times only the reference CPU module on the bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "diffusion Gvox·rep/s + HBM GB/s vs peak; bf16-field vs fp32 at stated FP64 err"
UNIT = "Gvox·rep/s"
FIELD_BYTES = {"f32": 4, "bf16": 2, "f16": 2, "f64": 8}
WORKLOADS = {
    # name: (shape, sigma, reps)
    "bone1024_s8_r100": ((1024, 1024, 1024), 8.0, 100),
    "bone512_s8_r100": ((512, 512, 512), 8.0, 100),
    "spheres128_s3_r10": ((128, 128, 128), 3.0, 10),
}
CPU_SAMPLE = ((512, 512, 512), 8.0, 1)  # bounded sample of the workload for the CPU arms
SECTIONS = ("e2e", "cfg0", "precision", "long", "batched", "out_of_core", "downstream", "cpu")

# DRAM bytes per voxel and repetition measured by ncu (dram__bytes_read.sum +
# dram__bytes_write.sum over the launches of one repetition, divided by the
# capture's voxels; captures larger than L2, traffic proportional to voxels):
# the FP32 CUDA-core passes on a 512^3 capture, the BF16 tensor-core passes on
# 256 x 1024 x 1024 (z, y and x passes as three kernels; the fused y + x kernel
# with the z pass).
NCU_BYTES_PER_VOXEL_REP = {
    ("f32", "separate"): (8237891584 + 8247201792 + 8356808704) / 2 ** 30,
    ("bf16", "separate"): (4136156160 + 4180311040 + 4272011263) / 2 ** 30,
    ("bf16", "fused"): (542214144 + 495355648 + 572188672 + 492044544) / 2 ** 28,
}


def alg_bytes_per_voxel_rep(field: str, mask: str) -> float:
    """Algorithmic HBM bytes per voxel and repetition: the field read and
    written once, the mask read once (2 s_field + s_mask)."""
    return 2 * FIELD_BYTES[field] + (1.0 if mask == "u8" else 0.125)


def parse_args():
    p = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--workload", choices=sorted(WORKLOADS), default="bone1024_s8_r100")
    p.add_argument("--field", choices=["f32", "bf16", "f16"], default="f32")
    p.add_argument("--quick", action="store_true", help="headline only: skip every section")
    p.add_argument("--sections", type=str, default=",".join(SECTIONS),
                   help="comma-separated sections to run after the headline (default: all): " + ",".join(SECTIONS))
    p.add_argument("--downstream-only", action="store_true",
                   help="run one diffusion of the workload, then only the downstream steps (field combination, "
                        "histograms, morphology, implant masks) on its output, and print their JSON object")
    p.add_argument("--shape", type=str, default=None,
                   help="override the workload's volume shape, e.g. 256x1024x1024 (profiling of smaller cases)")
    p.add_argument("--separate-passes", action="store_true",
                   help="16-bit fields: the headline step runs the y and x passes as two kernels instead of the "
                        "fused y + x tensor-core kernel")
    p.add_argument("--reps", type=int, default=None,
                   help="override the workload's repetition count (profiling of smaller cases)")
    p.add_argument("--ooc-shape", type=str, default="3456x3456x4096",
                   help="out-of-core section's volume, z x y x x")
    return p.parse_args()


_T0 = time.perf_counter()


def progress(msg: str) -> None:
    """One progress line on stderr (the JSON line alone goes to stdout)."""
    sys.stderr.write(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}\n")
    sys.stderr.flush()


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        rows = [l.strip().split(", ") for l in self.f if l.strip()]
        os.unlink(self.f.name)
        sm, reasons, mx = [], set(), None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 8:
                continue
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except ValueError:
                continue
            for name, val in zip(names, r[4:8]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(value: float, world: int, device: str) -> float:
    """The largest `value` over all ranks of the process group (every rank calls
    this at the same point); the identity on one rank."""
    if world <= 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, vox: int, reps: int, steps: int, seconds: float) -> float:
    """Gvox*rep/s of the whole job: every rank diffuses its own volume of `vox`
    voxels `steps` times; `seconds` is the slowest rank's time."""
    return world * vox * reps * steps / seconds / 1e9


def cpu_reference_time(shape, sigma, reps, repeats):
    """Time the reference OpenMP module (or the oracle port) on a synthetic sample."""
    import numpy as np
    import torch

    import oracle
    from maxibone_b200.kernels import gauss_kernel
    from maxibone_b200.synthetic import bone_implant_mask

    mask = bone_implant_mask(shape, seed=1, device="cpu").numpy()
    kernel = gauss_kernel(sigma).astype(np.float32)
    out = np.empty(shape, np.uint16)
    ref = oracle.reference_module("diffusion")
    kind = "reference" if ref is not None else "port"
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        if ref is not None:
            ref.diffusion(mask, kernel, out, reps)
        else:
            oracle.diffusion_in_memory(mask, kernel, reps)
        times.append(time.perf_counter() - t0)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    vox = shape[0] * shape[1] * shape[2]
    del torch
    return times, kind, cores, vox, (mask, kernel, out if ref is not None else None)


def run_reference_arm(args, rank):
    if rank != 0:
        return
    shape, sigma, reps = CPU_SAMPLE
    times, kind, cores, vox, _ = cpu_reference_time(shape, sigma, reps, args.warmup + args.steps)
    timed = times[args.warmup:]
    total = sum(timed)
    value = vox * reps * len(timed) / total / 1e9
    sample = (f"bone-implant mask {shape[0]}x{shape[1]}x{shape[2]}, sigma={sigma} (65 taps), R={reps} per step, "
              f"FP32, reference OpenMP module (oracle/_ref) via its pybind diffusion()")
    if kind == "port":
        sample = sample.replace("reference OpenMP module (oracle/_ref) via its pybind diffusion()",
                                "C restatement of the reference (oracle), OpenMP")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / len(timed) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload} (CPU sample: {shape[0]}^3, R={reps} per step)",
                   "parallelism": "host OpenMP"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def batched_section(device, torch, np, stream, reps=50):
    """64 uneven volumes, sigma in {2, 4, 8}, R = 50: one BF16 batch plan (one CUDA
    graph, one tensor-core launch per pass per group) vs per-volume FP32 launches."""
    from maxibone_b200.kernels import gauss_kernel
    from maxibone_b200.synthetic import batch_shapes, spheres_mask_torch

    specs = batch_shapes(64, seed=0)
    masks = [spheres_mask_torch(sh, fg, seed=i) for i, (sh, _, fg) in enumerate(specs)]
    kernels = [gauss_kernel(sig).astype(np.float32) for _, sig, _ in specs]
    outs = [torch.empty(sh, dtype=torch.uint16, device="cuda") for sh, _, _ in specs]
    fouts = [torch.empty(sh, dtype=torch.float32, device="cuda") for sh, _, _ in specs]
    vox = sum(int(np.prod(sh)) for sh, _, _ in specs)
    res = {"workload": "64 volumes, dims per axis from {96,128,192,256,384,512}, sigma from {2,4,8}, "
                       f"5-30% foreground spheres, R={reps}", "voxels": vox}
    plan = device.BatchPlan(masks, kernels, reps, outputs=outs, field="bf16", field_outs=fouts, autotune=True)
    res["plan"] = plan.describe()
    plan.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_t = 3
    e0.record(stream)
    for _ in range(n_t):
        plan.run()
    e1.record(stream)
    torch.cuda.synchronize()
    device.tensor_core_status()
    t_bf16 = e0.elapsed_time(e1) / n_t
    peak, _ = load_peaks()
    gbs = alg_bytes_per_voxel_rep("bf16", "bitpacked") * vox * reps / (t_bf16 / 1e3) / 1e9
    res["bf16_batch"] = {"value": vox * reps / (t_bf16 / 1e3) / 1e9, "unit": UNIT, "ms": t_bf16,
                         "hbm_gbs": gbs, "hbm_frac": gbs / peak,
                         "hbm_frac_definition": "V R (2 s_field + s_mask) / t / peak, 4.125 B per voxel-repetition"}
    # Accuracy of every volume against the FP64 form.
    errs, means = [], []
    for i in range(64):
        want = torch.empty(specs[i][0], dtype=torch.float64, device="cuda")
        device.diffuse(masks[i], kernels[i], reps, field="f64", field_out=want)
        d = (fouts[i].double() - want).abs_()
        errs.append(float(d.max().item()))
        means.append(float(d.mean().item()))
        del want, d
    res["bf16_batch"]["max_abs_err_vs_f64"] = max(errs)
    res["bf16_batch"]["mean_abs_err_vs_f64"] = sum(means) / len(means)
    res["bf16_batch"]["volumes_checked"] = len(errs)
    plan.close()
    # Per-volume FP32 launches (the plain form, one call per volume).
    ws = torch.empty(max(device.workspace_bytes(sh, "f32") for sh, _, _ in specs), dtype=torch.uint8, device="cuda")
    for i in range(2):
        device.diffuse(masks[i], kernels[i], reps, output=outs[i], field="f32", workspace=ws)
    torch.cuda.synchronize()
    e0.record(stream)
    for i in range(64):
        device.diffuse(masks[i], kernels[i], reps, output=outs[i], field="f32", workspace=ws)
    e1.record(stream)
    torch.cuda.synchronize()
    t_f32 = e0.elapsed_time(e1)
    res["f32_per_volume"] = {"value": vox * reps / (t_f32 / 1e3) / 1e9, "unit": UNIT, "ms": t_f32}
    res["speedup_bf16_batch_vs_f32_per_volume"] = t_f32 / t_bf16
    del masks, outs, fouts, ws
    torch.cuda.empty_cache()
    return res


def fields_section(torch, np, gauss_u16, stream):
    """The Gaussian + EDT field combination (the pipeline step after the
    diffusion) on the workload's uint16 output and a synthetic EDT-like field,
    against the reference's own CPU form of the step on a 256^3 sample."""
    import oracle
    from maxibone_b200.fields import combine_fields

    shape = tuple(gauss_u16.shape)
    vox = int(np.prod(shape))
    g = gauss_u16.view(torch.int16)
    zz = torch.arange(shape[0], device="cuda", dtype=torch.float32)[:, None, None]
    yy = torch.arange(shape[1], device="cuda", dtype=torch.float32)[None, :, None]
    xx = torch.arange(shape[2], device="cuda", dtype=torch.float32)[None, None, :]
    e = ((torch.sin(zz * 0.05) + torch.cos(yy * 0.03) + torch.sin(xx * 0.07) + 3.0) * 10000.0).to(torch.int32)
    e = e.to(torch.int16)
    out = torch.empty_like(g)
    combine_fields(g, e, out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_t = 5
    e0.record(stream)
    for _ in range(n_t):
        combine_fields(g, e, out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n_t
    peak, _ = load_peaks()
    alg = 14 * vox  # three passes reading both 2-byte fields, one 2-byte write
    res = {"workload": f"{shape[0]}x{shape[1]}x{shape[2]} uint16 Gaussian field (the diffusion output) + synthetic "
                       "uint16 EDT-like field", "value": vox / (ms / 1e3) / 1e9, "unit": "Gvox/s", "ms": ms,
           "hbm_gbs": alg / (ms / 1e3) / 1e9, "hbm_frac": alg / (ms / 1e3) / 1e9 / peak,
           "alg_bytes_per_voxel": 14, "timing": "CUDA events around 5 synchronous calls (two host read-backs each)"}
    # The reference's own form of the step on a bounded sample: its numpy operations with
    # the reference's compiled normalized_convert (oracle/_ref), else the oracle's numpy port.
    n = 256
    gs = gauss_u16[:n, :n, :n].cpu().numpy() if min(shape) >= n else gauss_u16.cpu().numpy()
    es = e.view(torch.uint16)[: gs.shape[0], : gs.shape[1], : gs.shape[2]].cpu().numpy()
    gs, es = np.ascontiguousarray(gs), np.ascontiguousarray(es)
    gen = oracle.reference_module("general")
    cyl = oracle.cylinder_mask(gs.shape[1], gs.shape[2])
    t0 = time.perf_counter()
    c = gs.astype(np.float32) / gs.max()
    c -= es.astype(np.float32) / es.max()
    c += np.abs(c.min())
    c /= c.max()
    c *= cyl
    if gen is not None:
        r = np.empty(c.shape, np.uint16)
        gen.normalized_convert(np.ascontiguousarray(c), r)
    else:
        r = oracle.normalized_convert_u16(c)
    r *= cyl
    cpu_s = time.perf_counter() - t0
    gpu_r = combine_fields(gs, es)
    res["cpu_baseline"] = {"value": gs.size / cpu_s / 1e9, "unit": "Gvox/s",
                           "kind": "reference" if gen is not None else "port",
                           "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                           "sample": f"{gs.shape[0]}x{gs.shape[1]}x{gs.shape[2]} crop, numpy steps of "
                                     "0975_combine_fields + normalized_convert, one call",
                           "gpu_equals_reference": bool(np.array_equal(gpu_r, r))}
    del e, out
    return res


def histogram_section(torch, np, mask, gauss_u16, stream):
    """The reference's histograms module (the pipeline's consumer of the diffusion
    field, src/processing_steps/1000_compute_histograms.py:470-472) on a synthetic
    uint16 tomogram made from the workload's mask: field_histogram against the
    diffusion output at half resolution with the pipeline's bins (2048 field x
    4096 voxel) and ranges, and axis_histograms (x, y, z, radial; 4096 bins) over
    the whole volume as one block.  Each against the reference's own compiled
    module on a bounded sample."""
    import oracle
    from maxibone_b200.histograms import axis_histograms, field_histogram

    shape = tuple(mask.shape)
    vox = int(np.prod(shape))
    g = torch.Generator(device="cuda").manual_seed(7)
    # Implant ~ 45000, bone-like ~ 12000-26000 with noise, background 0 in a quarter of the volume.
    noise = torch.randn(shape, generator=g, device="cuda") * 1500.0
    zz = torch.arange(shape[0], device="cuda", dtype=torch.float32)[:, None, None]
    base = 19000.0 + 7000.0 * torch.sin(zz * 0.01)
    vox_f = torch.where(mask.bool(), torch.full((), 45000.0, device="cuda"), base + noise)
    vox_f[:, :, : shape[2] // 4] = 0.0
    voxels = vox_f.clamp(0, 65535).to(torch.int32).to(torch.int16)
    del noise, vox_f, base
    field = gauss_u16.view(torch.int16)[::2, ::2, ::2].contiguous()
    vrange, frange = (1.0, 32000.0), (1.0, 65535.0)
    center = (shape[1] // 2, shape[2] // 2)
    n_r = int(np.sqrt((shape[2] // 2) ** 2 + (shape[1] // 2) ** 2)) + 1
    peak, _ = load_peaks()
    hist = oracle.reference_module("histograms")
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    n_t = 5

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n_t):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n_t

    out = {}
    bins = torch.zeros((2048, 4096), dtype=torch.int64, device="cuda")
    ms = timed(lambda: field_histogram(voxels, field, (0, 0, 0), bins, vrange, frange, 0))
    alg = 2.25 * vox  # each 2-byte voxel once, each 2-byte field sample once per 8 voxels
    res = {"workload": f"{shape[0]}x{shape[1]}x{shape[2]} synthetic uint16 tomogram vs the "
                       f"{tuple(field.shape)} half-resolution diffusion field, bins 2048x4096, vrange {vrange}",
           "value": vox / (ms / 1e3) / 1e9, "unit": "Gvox/s", "ms": ms,
           "counted_per_call": int(bins.sum().item()) // (n_t + 1),
           "hbm_gbs": alg / (ms / 1e3) / 1e9, "hbm_frac": alg / (ms / 1e3) / 1e9 / peak,
           "alg_bytes_per_voxel": 2.25,
           "timing": "CUDA events around 5 synchronous calls (host tables built and copied in each)"}
    n = 256
    vs = np.ascontiguousarray(voxels[:n, :n, :n].cpu().numpy().view(np.uint16))
    fs = np.ascontiguousarray(field[: n // 2, : n // 2, : n // 2].cpu().numpy().view(np.uint16))
    t0 = time.perf_counter()
    if hist is not None:
        ref = np.zeros((2048, 4096), np.uint64)
        hist.field_histogram(vs, fs, (0, 0, 0), ref, vrange, frange, 0)
    else:
        ref = oracle.field_histogram(vs, fs, (0, 0, 0), (2048, 4096), vrange, frange)
    cpu_s = time.perf_counter() - t0
    got = np.zeros((2048, 4096), np.uint64)
    field_histogram(vs, fs, (0, 0, 0), got, vrange, frange, 0)
    res["cpu_baseline"] = {"value": vs.size / cpu_s / 1e9, "unit": "Gvox/s",
                           "kind": "reference" if hist is not None else "port", "cores": cores,
                           "sample": f"{vs.shape} crop vs {fs.shape} field, one field_histogram call",
                           "gpu_equals_reference": bool(np.array_equal(got, ref))}
    out["field_histogram"] = res
    del bins

    axb = [torch.zeros((k, 4096), dtype=torch.int64, device="cuda") for k in (shape[2], shape[1], shape[0], n_r)]
    ms = timed(lambda: axis_histograms(voxels, (0, 0, 0), *axb, center, vrange, 0))
    res = {"workload": f"{shape[0]}x{shape[1]}x{shape[2]} synthetic uint16 tomogram as one block, x / y / z / "
                       f"radial histograms of 4096 bins (Nr {n_r}), vrange {vrange}",
           "value": vox / (ms / 1e3) / 1e9, "unit": "Gvox/s", "ms": ms,
           "counted_per_call": int(axb[0].sum().item()) // (n_t + 1),
           "hbm_gbs": 2 * vox / (ms / 1e3) / 1e9, "hbm_frac": 2 * vox / (ms / 1e3) / 1e9 / peak,
           "alg_bytes_per_voxel": 2,
           "timing": "CUDA events around 5 synchronous calls"}
    nz_s = 64
    vs = np.ascontiguousarray(voxels[:nz_s].cpu().numpy().view(np.uint16))
    shp = (shape[2], shape[1], shape[0], n_r)
    t0 = time.perf_counter()
    if hist is not None:
        ref = [np.zeros((k, 4096), np.uint64) for k in shp]
        hist.axis_histograms(vs, (0, 0, 0), *ref, center, vrange, 0)
    else:
        ref = oracle.axis_histograms(vs, (0, 0, 0), (shape[0], shape[1], shape[2]), 4096, n_r, center, vrange)
    cpu_s = time.perf_counter() - t0
    got = [np.zeros((k, 4096), np.uint64) for k in shp]
    axis_histograms(vs, (0, 0, 0), *got, center, vrange, 0)
    res["cpu_baseline"] = {"value": vs.size / cpu_s / 1e9, "unit": "Gvox/s",
                           "kind": "reference" if hist is not None else "port", "cores": cores,
                           "sample": f"{vs.shape} block (first {nz_s} planes), one axis_histograms call",
                           "gpu_equals_reference": all(np.array_equal(a, b) for a, b in zip(got, ref))}
    out["axis_histograms"] = res
    del voxels, field, axb
    return out


def morphology_section(torch, np, mask, stream):
    """The sphere morphology that prepares masks (src/lib/py/helpers.py:805-850 applies
    radius-16 spheres repeatedly) on the workload's mask: dilation with radius 16 in the
    uint8 form and in the bit-packed form, against the reference's compiled uint8
    module on a bounded sample."""
    import oracle
    from maxibone_b200 import morphology as mo

    shape = tuple(mask.shape)
    vox = int(np.prod(shape))
    r = 16
    n_t = 3

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n_t):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n_t

    m = (mask != 0).to(torch.uint8).contiguous()
    out = torch.empty_like(m)
    res = {}
    ms = timed(lambda: mo.dilate_3d_sphere(m, r, out))
    res["dilate_u8_r16"] = {"value": vox / (ms / 1e3) / 1e9, "unit": "Gvox/s", "ms": ms,
                            "foreground_after": float(out.float().mean().item())}
    words = None
    if shape[2] % 32 == 0:
        bits = torch.tensor([1 << (31 - b) for b in range(32)], device="cuda", dtype=torch.int64)
        w = torch.empty((shape[0], shape[1], shape[2] // 32), dtype=torch.int32, device="cuda")
        for z0 in range(0, shape[0], 64):  # pack in slabs to bound the int64 temporary
            t = (m[z0:z0 + 64].view(-1, shape[1], shape[2] // 32, 32).to(torch.int64) * bits).sum(-1)
            w[z0:z0 + 64] = (t - (t >= 2 ** 31).to(torch.int64) * 2 ** 32).to(torch.int32)
        words = w
        wout = torch.empty_like(words)
        ms = timed(lambda: mo.dilate_3d_sphere_bitpacked(words, r, wout))
        res["dilate_bitpacked_r16"] = {"value": vox / (ms / 1e3) / 1e9, "unit": "Gvox/s", "ms": ms}
    res["workload"] = (f"{shape[0]}x{shape[1]}x{shape[2]} bone-implant mask, sphere radius 16 (the radius "
                       "morph_3d applies repeatedly); timing: CUDA events around 3 synchronous calls")
    morph = oracle.reference_module("morphology")
    sample = (32, 128, 128)
    ms_ = m[: sample[0], : sample[1], : sample[2]].contiguous()
    sm = ms_.cpu().numpy()
    t0 = time.perf_counter()
    if morph is not None:
        ref = np.zeros(sample, np.uint8)
        morph.dilate_3d_sphere(sm, r, ref)
    else:
        ref = oracle.morphology_sphere(sm, r, True)
    cpu_s = time.perf_counter() - t0
    got = np.zeros(sample, np.uint8)
    mo.dilate_3d_sphere(sm, r, got)
    res["cpu_baseline"] = {"value": sm.size / cpu_s / 1e9, "unit": "Gvox/s",
                           "kind": "reference" if morph is not None else "port",
                           "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                           "sample": f"{sample} crop, one dilate_3d_sphere call with radius {r}",
                           "gpu_equals_reference": bool(np.array_equal(got, ref))}
    del m, out, words
    return res


def implant_section(torch, np, mask, stream):
    """The implant masks that feed the diffusion (compute_front_back_masks,
    src/processing_steps/0750_bone_region.py:62) on the workload's mask with a seeded
    frame of reference, against the reference's compiled geometry module on a bounded
    sample."""
    import oracle
    from maxibone_b200.geometry import compute_front_back_masks

    shape = tuple(mask.shape)
    vox = int(np.prod(shape))
    m = (mask != 0).to(torch.uint8).contiguous()
    rng = np.random.default_rng(5)
    E = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    UVWp = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    cm = torch.nonzero(m[:: 8]).to(torch.float64).mean(0).cpu().numpy() * np.array([8, 1, 1])
    cp = rng.normal(size=3) * 20
    outs = [torch.empty_like(m) for _ in range(4)]
    compute_front_back_masks(m, 1.875, E, cm, cp, UVWp, *outs)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_t = 3
    e0.record(stream)
    for _ in range(n_t):
        compute_front_back_masks(m, 1.875, E, cm, cp, UVWp, *outs)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / n_t
    peak, _ = load_peaks()
    alg = 7 * vox  # three reads of the 1-byte mask, four 1-byte masks written
    res = {"workload": f"{shape[0]}x{shape[1]}x{shape[2]} bone-implant mask, seeded frame of reference",
           "value": vox / (ms / 1e3) / 1e9, "unit": "Gvox/s", "ms": ms, "hbm_gbs": alg / (ms / 1e3) / 1e9,
           "hbm_frac": alg / (ms / 1e3) / 1e9 / peak, "alg_bytes_per_voxel": 7,
           "timing": "CUDA events around 3 synchronous calls"}
    geo = oracle.reference_module("geometry")
    sample = (64, 512, 512)
    sm = np.ascontiguousarray(m[: sample[0], : sample[1], : sample[2]].cpu().numpy())
    want = [np.empty(sm.shape, np.uint8) for _ in range(4)]
    t0 = time.perf_counter()
    if geo is not None:
        geo.compute_front_back_masks(sm, 1.875, E, cm, cp, UVWp, *want)
    else:
        want = list(oracle.implant_masks(sm, 1.875, E, cm, cp, UVWp))
    cpu_s = time.perf_counter() - t0
    got = [np.empty(sm.shape, np.uint8) for _ in range(4)]
    compute_front_back_masks(sm, 1.875, E, cm, cp, UVWp, *got)
    res["cpu_baseline"] = {"value": sm.size / cpu_s / 1e9, "unit": "Gvox/s",
                           "kind": "reference" if geo is not None else "port",
                           "cores": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
                           "sample": f"{sample} crop, one compute_front_back_masks call",
                           "gpu_equals_reference": all(np.array_equal(a, b) for a, b in zip(got, want))}
    del m, outs
    return res


def batched_plan_on_volume(device, torch, np, mask, kernel, reps, stream):
    """The BF16 batch plan (CUDA graph of persistent tensor-core launches, one per
    pass) over the workload's single volume: the batched form on the 1024^3 mask."""
    vox = int(mask.numel())
    out = torch.empty(tuple(mask.shape), dtype=torch.uint16, device="cuda")
    plan = device.BatchPlan([mask], [kernel], reps, outputs=[out], field="bf16")
    plan.run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_t = 2
    e0.record(stream)
    for _ in range(n_t):
        plan.run()
    e1.record(stream)
    torch.cuda.synchronize()
    device.tensor_core_status()
    plan.close()
    t = e0.elapsed_time(e1) / n_t
    peak, _ = load_peaks()
    gbs = alg_bytes_per_voxel_rep("bf16", "bitpacked") * vox * reps / (t / 1e3) / 1e9
    del out
    return {"value": vox * reps / (t / 1e3) / 1e9, "unit": UNIT, "ms": t, "hbm_gbs": gbs, "hbm_frac": gbs / peak}


def sampled(local_rank, fn):
    """Runs fn() while nvidia-smi samples the clocks; returns (result, clocks)."""
    sampler = ClockSampler(local_rank)
    try:
        res = fn()
    finally:
        clocks = sampler.stop()
    return res, clocks


class PinnedArray:
    """A numpy array page-locked with cudaHostRegister: exactly its own size
    (torch's pinned allocator rounds every allocation up to a power of two,
    which turns 43 + 87 GB into 64 + 128 GB)."""

    def __init__(self, torch, np, shape, dtype):
        self.torch = torch
        self.a = np.empty(shape, dtype)
        self.ptr = self.a.ctypes.data
        rc = int(torch.cuda.cudart().cudaHostRegister(self.ptr, self.a.nbytes, 0))
        if rc != 0:
            raise MemoryError(f"cudaHostRegister of {self.a.nbytes} bytes failed ({rc})")

    def close(self):
        if self.ptr:
            self.torch.cuda.cudart().cudaHostUnregister(self.ptr)
            self.ptr = 0
            self.a = None


def out_of_core_section(torch, np, shape, reps=20):
    """cfg4: a bone-implant mask larger than the device in pinned host memory
    (3456 x 3456 x 4096, z x y x x, 49 GB), sigma 8, R = 20, BF16 field, through
    the out-of-core form end to end: one timed call from host mask to host
    uint16 output, PCIe copies included.  The planner chooses slab depth and
    plan from the free device memory.  If the host lacks the RAM for the pinned
    mask and output, the z extent is reduced and the reason recorded."""
    import ctypes

    import psutil

    from maxibone_b200 import _lib, device
    from maxibone_b200.diffusion import diffusion_out_of_core
    from maxibone_b200.kernels import gauss_kernel
    from maxibone_b200.synthetic import bone_implant_mask

    nz, ny, nx = shape
    avail = psutil.virtual_memory().available
    note = None
    need = 3 * nz * ny * nx  # uint8 mask + uint16 output
    if need > 0.75 * avail:
        nz_fit = max(64, int(0.75 * avail / (3 * ny * nx)) // 64 * 64)
        note = (f"host RAM {avail / 1e9:.0f} GB available: z reduced from {nz} to {nz_fit} "
                f"(the pinned mask and output need 3 bytes per voxel)")
        nz = min(nz, nz_fit)
    shape = (nz, ny, nx)
    vox = nz * ny * nx
    kernel = gauss_kernel(8.0).astype(np.float32)
    t0 = time.perf_counter()
    pin_m = PinnedArray(torch, np, shape, np.uint8)
    pin_o = PinnedArray(torch, np, shape, np.uint16)
    host_m = torch.from_numpy(pin_m.a)
    t_alloc = time.perf_counter() - t0
    t0 = time.perf_counter()
    chunk = 128
    for z0 in range(0, nz, chunk):  # generate on the GPU in chunks of planes
        z1 = min(nz, z0 + chunk)
        host_m[z0:z1].copy_(bone_implant_mask((z1 - z0, ny, nx), seed=z0, implant_radius=120.0 * ny / 1024,
                                              device="cuda"))
    torch.cuda.synchronize()
    t_gen = time.perf_counter() - t0
    s_, k_, r_ = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    _lib.check(_lib.lib().maxi_out_of_core_plan(nz, ny, nx, 0, kernel.shape[0], reps, _lib.FIELD_TYPES["bf16"], 0, 0,
                                                ctypes.byref(s_), ctypes.byref(k_), ctypes.byref(r_)))
    m_np, o_np = pin_m.a, pin_o.a
    device.profile_enable(True)
    device.profile_read()
    t0 = time.perf_counter()
    diffusion_out_of_core(m_np, kernel, o_np, (0, ny, nx), reps, field="bf16")
    dt = time.perf_counter() - t0
    prof = device.profile_read()
    device.profile_enable(False)
    kernel_s = sum(v[0] for v in prof.values()) / 1e3
    S, k = s_.value, k_.value
    r = kernel.shape[0] // 2
    n_slabs = -(-nz // S)
    halo = min(nz, k * r)
    computed = 0
    for sl in range(n_slabs):
        z0, z1 = sl * S, min(nz, (sl + 1) * S)
        cuts = (z0 > 0) + (z1 < nz)
        computed += (z1 - z0) * reps + cuts * r * k * (k + 1) // 2 * (-(-reps // k))
    zs = np.linspace(0, nz - 1, 8).astype(int)
    mask_exact = all(bool(np.all(o_np[z][m_np[z] > 0] == 65535)) for z in zs)
    res = {"workload": f"{nz}x{ny}x{nx} (z x y x x) bone-implant mask in pinned host memory, sigma 8 (65 taps), "
                       f"R={reps}, BF16 field, uint16 output to pinned host memory", "voxels": vox,
           "value": vox * reps / dt / 1e9, "unit": UNIT, "seconds": dt,
           "plan": {"slab_planes": S, "slabs": n_slabs, "reps_per_round": k, "halo_planes": halo,
                    "resident_bitpacked_mask": bool(r_.value),
                    "compute_redundancy": computed / (nz * reps)},
           "h2d_bytes": vox, "d2h_bytes": 2 * vox,
           "mask_voxels_exact_on_sampled_planes": mask_exact,
           "timing": "host clock around one synchronous out-of-core call (mask upload, slabs, downloads)",
           "kernel_seconds": kernel_s,
           "kernel_seconds_definition": "summed CUDA-event time of the library's kernels in the call (they overlap "
                                        "the host copies; the rest of `seconds` is copy time not hidden)",
           "kernels": {k: {"launches": v[1], "ms": v[0]} for k, v in prof.items()},
           "setup_seconds": {"pinned_allocation": t_alloc, "mask_generation": t_gen}}
    if note:
        res["note"] = note
    del host_m, m_np, o_np
    pin_m.close()
    pin_o.close()
    return res


def form_runs(device, torch, np, mask, kernel, reps, forms, stream, shape=None, n_t=2, packed=False):
    """Runs each (name, field, opts) form: a timed run (CUDA events, n_t calls,
    uint16 output only) and one run writing the field for the errors against
    the FP64 form (and the FP32 form where run).  mask: uint8 tensor, or
    bit-packed words with `shape`."""
    peak, _ = load_peaks()
    vox = int(np.prod(shape if shape is not None else tuple(mask.shape)))
    shp = shape if shape is not None else tuple(mask.shape)
    f64 = torch.empty(shp, dtype=torch.float64, device="cuda")
    device.diffuse(mask, kernel, reps, field="f64", field_out=f64, shape=shape)
    out = torch.empty(shp, dtype=torch.uint16, device="cuda")
    res, f32_field = {}, None
    for name, form, opts in forms:
        fo = torch.empty(shp, dtype=torch.float32, device="cuda")
        w = torch.empty(device.workspace_bytes(shp, form), dtype=torch.uint8, device="cuda")
        device.diffuse(mask, kernel, reps, output=out, field=form, field_out=fo, workspace=w, shape=shape, **opts)
        path = device.last_path()
        torch.cuda.synchronize()
        device.profile_enable(True)
        device.profile_read()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n_t):
            device.diffuse(mask, kernel, reps, output=out, field=form, workspace=w, shape=shape, **opts)
        e1.record(stream)
        torch.cuda.synchronize()
        prof = device.profile_read()
        device.profile_enable(False)
        device.tensor_core_status()
        t_ms = e0.elapsed_time(e1) / n_t
        err = (fo.double() - f64).abs_()
        b_alg = alg_bytes_per_voxel_rep(form, "bitpacked" if packed else "u8")
        gbs = b_alg * vox * reps / (t_ms / 1e3) / 1e9
        entry = {"value": vox * reps / (t_ms / 1e3) / 1e9, "unit": UNIT, "field": form, **opts,
                 "ms_per_call": t_ms, "hbm_gbs": gbs, "hbm_frac": gbs / peak, "alg_bytes_per_voxel_rep": b_alg,
                 "max_abs_err_vs_f64": float(err.max().item()), "mean_abs_err_vs_f64": float(err.mean().item()),
                 "mask_voxels_exact": bool((out.view(torch.int16)[mask > 0] == -1).all().item())
                 if shape is None else None,
                 "path_bits": path, "per_kind_ms": {k: v[0] / v[1] for k, v in prof.items()},
                 "launches_per_call": sum(v[1] for v in prof.values()) // n_t}
        if form == "f32" and not opts:
            f32_field = fo
        elif f32_field is not None:
            entry["max_abs_err_vs_f32"] = float((fo - f32_field).abs_().max().item())
        res[name] = entry
        del err, w
        if fo is not f32_field:
            del fo
        torch.cuda.empty_cache()
    del f64, out, f32_field
    torch.cuda.empty_cache()
    return res


PRECISION_FORMS = [
    ("f32", "f32", {}),
    ("bf16", "bf16", {}),
    ("bf16_split_coefficients", "bf16", {"split_coefficients": True}),
    ("bf16_separate_passes", "bf16", {"fuse_passes": False}),
    ("f16", "f16", {}),
    ("f16_split_coefficients", "f16", {"split_coefficients": True}),
    ("bf16_nearest", "bf16", {"error_feedback": False}),
    ("bf16_cuda_cores", "bf16", {"tensor_cores": False}),
]


def precision_section(device, torch, np, mask, kernel, reps, stream):
    """cfg2 at R = 100: the workload's mask bit-packed (1 bit per voxel), the
    FP32 field and the 16-bit field forms, each with its error against the FP64
    form and the FP32 form."""
    shape = tuple(mask.shape)
    packed = device.bitpack(mask)
    res = form_runs(device, torch, np, packed, kernel, reps, PRECISION_FORMS, stream, shape=shape, packed=True)
    for name in res:  # mask exactness on the uint8 view of the same runs
        res[name].pop("mask_voxels_exact", None)
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    for form in ("bf16", "f16"):
        device.diffuse(packed, kernel, reps, output=out, field=form, shape=shape)
        res[form]["mask_voxels_exact"] = bool((out.view(torch.int16)[mask > 0] == -1).all().item())
    del packed, out
    return res


def long_section(device, torch, np, mask, kernel, stream):
    """cfg2's R = 500 runs (BF16 and FP16, both coefficient forms) and the
    sigma = 32 (radius 128, 257 taps) case at R = 20: the FP32 CUDA-core
    stencil and the BF16 CUDA-core passes against the BF16 / FP16 banded-Toeplitz
    tensor-core passes, each against the FP64 form."""
    from maxibone_b200.kernels import gauss_kernel

    shape = tuple(mask.shape)
    packed = device.bitpack(mask)
    res = {"r500": form_runs(device, torch, np, packed, kernel, 500,
                             [("bf16", "bf16", {}), ("bf16_split_coefficients", "bf16", {"split_coefficients": True}),
                              ("f16", "f16", {})], stream, shape=shape, n_t=1, packed=True)}
    k32 = gauss_kernel(32.0).astype(np.float32)
    res["sigma32_r20"] = form_runs(device, torch, np, packed, k32, 20,
                                   [("f32_cuda_cores", "f32", {}), ("bf16_tensor_cores", "bf16", {}),
                                    ("f16_tensor_cores", "f16", {}),
                                    ("bf16_cuda_cores", "bf16", {"tensor_cores": False})],
                                   stream, shape=shape, n_t=1, packed=True)
    for part in res.values():
        for entry in part.values():
            entry.pop("mask_voxels_exact", None)
    res["sigma32_r20"]["kernel_size"] = int(k32.shape[0])
    del packed
    return res


def cfg0_section(device, torch, np, stream):
    """cfg0: the 128^3 union of 40 spheres, sigma 3 (25 taps), R = 10, FP32
    field: device rate, the reference-facing host call, and the reference
    module on the same input (full run, median of 3) with the uint16 outputs
    compared."""
    import oracle
    from maxibone_b200.diffusion import diffusion
    from maxibone_b200.kernels import gauss_kernel
    from maxibone_b200.synthetic import spheres_mask

    shape, reps = (128, 128, 128), 10
    mask_np = spheres_mask(shape, 40, (4, 20), seed=0)
    kernel = gauss_kernel(3.0).astype(np.float32)
    vox = int(np.prod(shape))
    m = torch.from_numpy(mask_np).cuda()
    out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    ws = torch.empty(device.workspace_bytes(shape, "f32"), dtype=torch.uint8, device="cuda")
    for _ in range(3):
        device.diffuse(m, kernel, reps, output=out, workspace=ws)
    torch.cuda.synchronize()
    n_t = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n_t):
        device.diffuse(m, kernel, reps, output=out, workspace=ws)
    e1.record(stream)
    torch.cuda.synchronize()
    t_ms = e0.elapsed_time(e1) / n_t
    host_out = np.empty(shape, np.uint16)
    diffusion(mask_np, kernel, host_out, reps)
    tw = time.perf_counter()
    for _ in range(5):
        diffusion(mask_np, kernel, host_out, reps)
    e2e_s = (time.perf_counter() - tw) / 5
    res = {"workload": "128^3 union of 40 spheres (radii 4-20, seed 0), sigma 3 (25 taps), R=10, FP32 field",
           "foreground": float(mask_np.mean()), "value": vox * reps / (t_ms / 1e3) / 1e9, "unit": UNIT,
           "ms_per_call": t_ms,
           "e2e": {"value": vox * reps / e2e_s / 1e9, "unit": UNIT, "ms_per_call": e2e_s * 1e3,
                   "timing": "host clock around 5 synchronous drop-in diffusion() calls (numpy in / out)"}}
    ref = oracle.reference_module("diffusion")
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    if ref is not None:
        want = np.empty(shape, np.uint16)
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            ref.diffusion(mask_np, kernel, want, reps)
            times.append(time.perf_counter() - t0)
        d = np.abs(host_out.astype(np.int32) - want.astype(np.int32))
        res["cpu_baseline"] = {"value": vox * reps / statistics.median(times) / 1e9, "unit": UNIT, "cores": cores,
                               "kind": "reference", "sample": "the whole cfg0 call, median of 3"}
        res["vs_reference_u16"] = {"max_lsb": int(d.max()), "voxels_differing": int((d > 0).sum())}
    del m, out, ws
    return res


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank)

    import datetime

    import numpy as np
    import torch
    import torch.distributed as dist

    from maxibone_b200 import _lib, device
    from maxibone_b200.diffusion import diffusion
    from maxibone_b200.kernels import gauss_kernel
    from maxibone_b200.synthetic import bone_implant_mask, spheres_mask

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
        # A collective over every rank first, so that the communicator exists
        # before the split's first grouped point-to-point exchange.
        dist.barrier()
    shape, sigma, reps = WORKLOADS[args.workload]
    if args.shape:
        shape = tuple(int(v) for v in args.shape.lower().split("x"))
    if args.reps is not None:
        reps = args.reps
    nz, ny, nx = shape
    vox = nz * ny * nx
    kernel = gauss_kernel(sigma).astype(np.float32)
    radius = kernel.shape[0] // 2
    if args.workload.startswith("spheres"):
        mask = torch.from_numpy(spheres_mask(shape, 40, (4, 20), seed=0)).cuda()
    else:
        mask = bone_implant_mask(shape, seed=0, device="cuda")
    fg = float(mask.float().mean().item())
    stream = torch.cuda.current_stream()
    split = None
    if world > 1:
        # One volume split into z-slabs over the ranks (strong scaling): every rank
        # holds its slab with the halos of its rounds and exchanges halo planes with
        # its neighbours between rounds (NCCL P2P over NVLink).
        from maxibone_b200.zsplit import diffuse_split, library_step, split_plan
        split = split_plan(nz, world, radius, reps)
        e0, e1 = split.extended(rank)
        z0, z1 = split.bounds[rank]
        mask = mask[e0:e1].contiguous()
        out = torch.empty((z1 - z0, ny, nx), dtype=torch.uint16, device="cuda")
        ws = None
        slab_step = library_step(args.field)

        def step(field=args.field, output=out, workspace=None, field_out=None):
            diffuse_split(mask, kernel, split, rank, world, slab_step, output=output)
    else:
        out = torch.empty(shape, dtype=torch.uint16, device="cuda")
        ws = torch.empty(device.workspace_bytes(shape, args.field), dtype=torch.uint8, device="cuda")

        def step(field=args.field, output=out, workspace=ws, field_out=None):
            device.diffuse(mask, kernel, reps, output=output, field=field, workspace=workspace, field_out=field_out,
                           fuse_passes=not args.separate_passes)

    def barrier():
        if world > 1:
            dist.barrier()

    if args.downstream_only:
        step()
        torch.cuda.synchronize()
        if rank == 0:
            print(json.dumps({"workload": args.workload, "shape": list(shape), "field": args.field,
                              "fields": {"combine_fields": fields_section(torch, np, out, stream),
                                         **histogram_section(torch, np, mask, out, stream)},
                              "morphology": morphology_section(torch, np, mask, stream),
                              "implant_masks": implant_section(torch, np, mask, stream)}), flush=True)
        return

    for _ in range(args.warmup):
        step()
    path = device.last_path()
    torch.cuda.synchronize()
    barrier()
    device.profile_enable(True)
    device.profile_read()
    sampler = ClockSampler(local_rank)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0.record(stream)
    for _ in range(args.steps):
        step()
    t1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    prof = device.profile_read()
    device.profile_enable(False)
    barrier()
    ms_local = t0.elapsed_time(t1)
    ms = max_over_ranks(ms_local, world, "cuda")
    # split: the ranks share one volume (its voxels counted once); otherwise each
    # rank diffuses its own volume
    value = whole_job_rate(1 if split else world, vox, reps, args.steps, ms / 1e3)
    launches = sum(c for _, c in prof.values())

    # Roofline: the repetition's algorithmic bytes V (2 s_field + s_mask) over its
    # device time (this GPU's volume and time), against the measured HBM bandwidth.
    peak, peak_kind = load_peaks()
    s = FIELD_BYTES[args.field]
    b_alg = alg_bytes_per_voxel_rep(args.field, "u8")
    rep_ms = ms_local / (args.steps * reps)
    vox_local = int(mask.numel()) if split else vox  # this GPU's voxels (a split rank's slab with halos)
    achieved = b_alg * vox_local / (rep_ms / 1e3) / 1e9
    fused = bool(path & _lib.PATH_FUSED_YX)
    per_voxel_traffic = NCU_BYTES_PER_VOXEL_REP.get((args.field, "fused" if fused else "separate"))
    kernel_bytes = {"z": 2 * s, "y": 2 * s, "x": 2 * s + 0.125, "x_final": s + 0.125 + 2, "yx": 2 * s + 0.125,
                    "init": 0.125 + s}
    per_kernel = {}
    for kind, (k_ms, k_n) in prof.items():
        if kind in kernel_bytes:
            gbs = kernel_bytes[kind] * vox_local / (k_ms / k_n / 1e3) / 1e9
            per_kernel[kind] = {"launches": k_n, "ms_per_launch": k_ms / k_n, "alg_bytes_per_launch":
                                kernel_bytes[kind] * vox_local, "gbs": gbs, "frac": gbs / peak}
    dom = max(prof, key=lambda k: prof[k][0])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": per_voxel_traffic * vox if per_voxel_traffic else None,
                "unit_of_work": f"one repetition (z, y and x passes with re-illumination) over {nz}x{ny}x{nx}",
                "alg_bytes_per_voxel_rep": b_alg,
                "alg_bytes_definition": "2 s_field + s_mask: the field read and written once, the uint8 mask read "
                                        "once, per voxel and repetition",
                "ms_per_repetition": rep_ms, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic_definition": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one repetition's "
                                      "launches, scaled from a capture larger than L2 by voxel count",
                "dominant_kernel": {"kind": dom, **per_kernel.get(dom, {})}, "per_kernel": per_kernel}
    if args.field == "f32":
        flop = 2 * 3 * (2 * radius + 1) * vox
        roofline["fp32_pipe"] = {
            "achieved_tflops": flop / (rep_ms / 1e3) / 1e12,
            "peak_tflops_computed": 148 * 128 * 2 * clocks["sm_mhz"] * 1e6 / 1e12 if clocks else None,
            "peak_source": "computed, not measured: 148 SMs x 128 FP32 lanes x 2 flop x the median SM clock",
            "note": "the direct FP32 stencil at radius 32 is bound by the FP32 pipe: 2 x 65 flop per 8 B of "
                    "field traffic per pass"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if split else "weak",
        "vs_baseline": None, "dtype": args.field, "data": "synthetic (seeded bone+implant mask, random-init)",
        "config": {"workload": args.workload + (f" (shape override {args.shape})" if args.shape else "")
                   + (f" (repetitions override {args.reps})" if args.reps is not None else ""),
                   "shape": list(shape), "sigma": sigma, "kernel_size": int(2 * radius + 1),
                   "reps": reps, "field": args.field, "separate_passes": bool(args.separate_passes), "mask": "u8",
                   "foreground": round(fg, 4),
                   "parallelism": (f"one volume split into {world} z-slabs (one per rank), halo planes exchanged "
                                   f"every {split.k} repetitions by NCCL P2P" if split else
                                   f"{world} independent volumes (one per rank)"),
                   "l2": "inputs larger than L2 (field %d MiB per buffer)" % (s * vox >> 20),
                   "path_bits": path},
        "gpu_launches": launches, "roofline": roofline, "clocks": clocks,
    }
    # the sections describe one GPU's forms: a split run reports the headline only
    sections = [] if (args.quick or split) else [x for x in args.sections.split(",") if x]
    if split and not args.quick:
        # End to end at N GPUs: each rank uploads its mask slab from pinned host
        # memory, runs the split, and downloads its core planes of the output.
        host_mask = torch.empty(tuple(mask.shape), dtype=torch.uint8, pin_memory=True)
        host_mask.copy_(mask)
        host_out = torch.empty(tuple(out.shape), dtype=torch.int16, pin_memory=True)

        def e2e_call():
            mask.copy_(host_mask, non_blocking=True)
            step()
            host_out.view(torch.uint16).copy_(out, non_blocking=True)
            torch.cuda.synchronize()

        e2e_call()
        barrier()
        tw = time.perf_counter()
        n_e2e = max(1, min(args.steps, 2))
        for _ in range(n_e2e):
            e2e_call()
        e2e_s = max_over_ranks(time.perf_counter() - tw, world, "cuda")
        line["e2e"] = {"value": whole_job_rate(1, vox, reps, n_e2e, e2e_s), "unit": UNIT,
                       "h2d_bytes_per_step": int(mask.numel()), "d2h_bytes_per_step": 2 * int(out.numel()),
                       "steps": n_e2e, "timing": "host clock around upload, split run and download (max over ranks); "
                                                 "bytes per rank"}
        del host_mask, host_out

    if "e2e" in sections:
        progress("section e2e")
        # End to end through the reference-facing call: numpy in, numpy out, from
        # pinned host memory and from pageable host memory (maxibone's callers
        # pass np.empty arrays).
        host_mask = torch.empty(shape, dtype=torch.uint8, pin_memory=True)
        host_mask.copy_(mask)
        host_out = torch.empty(shape, dtype=torch.int16, pin_memory=True)
        m_np, o_np = host_mask.numpy(), host_out.numpy().view(np.uint16)
        del ws
        torch.cuda.empty_cache()
        e2e = {}
        for kind, (mi, oi) in (("pinned", (m_np, o_np)),
                               ("pageable", (np.array(m_np), np.empty(shape, np.uint16)))):
            diffusion(mi, kernel, oi, reps)  # warm-up
            n_e2e = max(1, min(args.steps, 2))
            barrier()
            tw = time.perf_counter()
            for _ in range(n_e2e):
                diffusion(mi, kernel, oi, reps)
            e2e_s = max_over_ranks(time.perf_counter() - tw, world, "cuda")
            e2e[kind] = {"value": whole_job_rate(world, vox, reps, n_e2e, e2e_s), "steps": n_e2e,
                         "ms_per_call": e2e_s / n_e2e * 1e3}
        line["e2e"] = {"value": e2e["pinned"]["value"], "unit": UNIT, "h2d_bytes_per_step": vox,
                       "d2h_bytes_per_step": 2 * vox, "steps": e2e["pinned"]["steps"],
                       "pageable": e2e["pageable"],
                       "timing": "host clock around the synchronous drop-in diffusion() call (max over ranks); the "
                                 "call allocates and frees its device buffers, as the reference does"}
        del host_mask, host_out
        ws = None
    else:
        ws = None
        torch.cuda.empty_cache()

    if "precision" in sections:
        progress("section precision")
        res, ck = sampled(local_rank, lambda: precision_section(device, torch, np, mask, kernel, reps, stream))
        res["clocks"] = ck
        res["workload"] = (f"{nz}x{ny}x{nx} bone-implant mask bit-packed (1 bit per voxel), sigma {sigma}, R={reps}; "
                           "hbm_frac = V R (2 s_field + 1/8) / t / peak")
        line["precision"] = res
        line["bf16_vs_f32"] = {"speedup": res["bf16"]["value"] / res["f32"]["value"],
                               "bf16_hbm_frac": res["bf16"]["hbm_frac"],
                               "bf16_max_abs_err_vs_f64": res["bf16"]["max_abs_err_vs_f64"],
                               "bf16_split_coefficients_speedup": res["bf16_split_coefficients"]["value"] /
                               res["f32"]["value"],
                               "bf16_split_coefficients_max_abs_err_vs_f64":
                                   res["bf16_split_coefficients"]["max_abs_err_vs_f64"]}
    if "long" in sections:
        progress("section long")
        res, ck = sampled(local_rank, lambda: long_section(device, torch, np, mask, kernel, stream))
        res["clocks"] = ck
        line["long"] = res
    if "cfg0" in sections:
        progress("section cfg0")
        res, ck = sampled(local_rank, lambda: cfg0_section(device, torch, np, stream))
        res["clocks"] = ck
        line["cfg0"] = res
    if "downstream" in sections:
        progress("section downstream")
        out_u16 = torch.empty(shape, dtype=torch.uint16, device="cuda")
        device.diffuse(mask, kernel, reps, output=out_u16)
        line["fields"] = {"combine_fields": fields_section(torch, np, out_u16, stream),
                          **histogram_section(torch, np, mask, out_u16, stream)}
        line["morphology"] = morphology_section(torch, np, mask, stream)
        line["implant_masks"] = implant_section(torch, np, mask, stream)
        del out_u16
    if "batched" in sections:
        progress("section batched")
        res, ck = sampled(local_rank, lambda: batched_section(device, torch, np, stream))
        res["clocks"] = ck
        line["batched"] = res
        res["bf16_plan_on_workload_volume"] = bv = batched_plan_on_volume(device, torch, np, mask, kernel, reps,
                                                                          stream)
        if "precision" in line:
            bv["speedup_vs_f32"] = bv["value"] / line["precision"]["f32"]["value"]
    torch.cuda.empty_cache()
    if "out_of_core" in sections and world == 1:
        progress("section out_of_core")
        ooc_shape = tuple(int(v) for v in args.ooc_shape.lower().split("x"))
        del mask
        torch.cuda.empty_cache()
        res, ck = sampled(local_rank, lambda: out_of_core_section(torch, np, ooc_shape))
        res["clocks"] = ck
        line["out_of_core"] = res
        mask = None

    if "cpu" in sections and rank == 0 and world == 1:
        progress("section cpu")
        cshape, csig, creps = CPU_SAMPLE
        times, kind, cores, cvox, (cmask, ckernel, cref) = cpu_reference_time(cshape, csig, creps, 2)
        line["cpu_baseline"] = {"value": cvox * creps / min(times) / 1e9, "unit": UNIT, "cores": cores,
                                "kind": kind,
                                "sample": f"bone-implant mask {cshape[0]}^3, sigma={csig} (65 taps), R={creps}, "
                                          f"best of 2 calls"}
        if cref is not None:
            # The FP32 path against the reference module's own uint16 output on the sample.
            gout = torch.empty(cshape, dtype=torch.uint16, device="cuda")
            device.diffuse(torch.from_numpy(cmask).cuda(), ckernel, creps, output=gout, field="f32")
            d = np.abs(gout.cpu().numpy().astype(np.int32) - cref.astype(np.int32))
            line["cpu_baseline"]["f32_vs_reference_u16"] = {"max_lsb": int(d.max()),
                                                            "voxels_differing": int((d > 0).sum())}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
