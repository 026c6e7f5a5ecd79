"""Seeded synthetic masks standing in for maxibone's implant masks.

The reference's tomograms are not available, so the workloads use masks with
the stated shapes and foreground fractions:

* ``spheres_mask``: union of random spheres (radii uniform in a range, centres
  uniform in the box), numpy ``default_rng(seed)``.
* ``bone_implant_mask``: a solid cylinder along z through the centre (the
  implant) plus thresholded two-octave value noise (trabecular-like sheets and
  struts), topped up to a target foreground fraction.  Built with torch on the
  given device so a 1024^3 mask takes well under a second on a GPU.
"""
from __future__ import annotations

import numpy as np


def spheres_mask(shape, n_spheres: int = 40, r_range=(4, 20), seed: int = 0) -> np.ndarray:
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0, 1, size=(n_spheres, 3)) * np.array([nz, ny, nx])
    radii = rng.uniform(r_range[0], r_range[1], size=n_spheres)
    mask = np.zeros(shape, dtype=np.uint8)
    for (cz, cy, cx), r in zip(centres, radii):
        z0, z1 = max(0, int(cz - r)), min(nz, int(cz + r) + 1)
        y0, y1 = max(0, int(cy - r)), min(ny, int(cy + r) + 1)
        x0, x1 = max(0, int(cx - r)), min(nx, int(cx + r) + 1)
        if z0 >= z1 or y0 >= y1 or x0 >= x1:
            continue
        z = np.arange(z0, z1)[:, None, None] - cz
        y = np.arange(y0, y1)[None, :, None] - cy
        x = np.arange(x0, x1)[None, None, :] - cx
        mask[z0:z1, y0:y1, x0:x1] |= (z * z + y * y + x * x <= r * r).astype(np.uint8)
    return mask


def random_mask(shape, fraction: float, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return (rng.random(shape) < fraction).astype(np.uint8)


def bone_implant_mask(shape, seed: int = 0, foreground: float = 0.25, implant_radius: float = 120.0,
                      device="cpu"):
    """uint8 torch tensor [nz, ny, nx] on `device`: implant cylinder + noise structures."""
    import torch
    import torch.nn.functional as F

    nz, ny, nx = shape
    g = torch.Generator(device="cpu").manual_seed(seed)
    field = None
    for cells, weight in ((16, 1.0), (48, 0.5)):
        coarse = torch.rand((1, 1, max(2, nz * cells // 1024 + 2), max(2, ny * cells // 1024 + 2),
                             max(2, nx * cells // 1024 + 2)), generator=g)
        coarse = coarse.to(device=device, dtype=torch.float32)
        up = F.interpolate(coarse, size=(nz, ny, nx), mode="trilinear", align_corners=True)[0, 0]
        field = up * weight if field is None else field.add_(up, alpha=weight)
        del up
    # Ridge structure: voxels near the noise's median level form thin sheets.
    flat = field.reshape(-1)
    idx = torch.randint(0, flat.numel(), (1 << 20,), generator=g).to(device)
    sample = flat[idx]
    median = sample.median()
    dist = (field - median).abs_()
    del field
    yy = torch.arange(ny, device=device, dtype=torch.float32)[:, None] - (ny - 1) / 2
    xx = torch.arange(nx, device=device, dtype=torch.float32)[None, :] - (nx - 1) / 2
    cyl = (yy * yy + xx * xx) <= implant_radius * implant_radius
    cyl_frac = cyl.float().mean().item()
    want = max(0.0, (foreground - cyl_frac) / max(1e-9, 1.0 - cyl_frac))
    thr = torch.quantile(dist.reshape(-1)[idx].float(), want).item() if want > 0 else -1.0
    mask = (dist <= thr)
    del dist
    mask |= cyl[None, :, :]
    return mask.to(torch.uint8)


def spheres_mask_torch(shape, foreground: float, seed: int = 0, device="cuda", r_frac=(0.04, 0.12)):
    """uint8 torch tensor: random spheres (radius r_frac x the smallest extent)
    placed until the expected covered fraction reaches `foreground`."""
    import math

    import torch

    nz, ny, nx = shape
    g = np.random.default_rng(seed)
    vol = nz * ny * nx
    rmin, rmax = (f * min(shape) for f in r_frac)
    mean_v = 4.0 / 3.0 * math.pi * ((rmin + rmax) / 2) ** 3
    count = max(1, int(-math.log(max(1e-6, 1.0 - foreground)) * vol / mean_v))
    if count > 200:  # fewer, larger spheres with the same expected coverage
        scale = (count / 200) ** (1.0 / 3.0)
        rmin, rmax, count = rmin * scale, rmax * scale, 200
    mask = torch.zeros(shape, dtype=torch.bool, device=device)
    zz = torch.arange(nz, device=device, dtype=torch.float32)
    yy = torch.arange(ny, device=device, dtype=torch.float32)
    xx = torch.arange(nx, device=device, dtype=torch.float32)
    for _ in range(count):
        cz, cy, cx = g.uniform(0, nz), g.uniform(0, ny), g.uniform(0, nx)
        r = g.uniform(rmin, rmax)
        z0, z1 = max(0, int(cz - r)), min(nz, int(cz + r) + 1)
        y0, y1 = max(0, int(cy - r)), min(ny, int(cy + r) + 1)
        x0, x1 = max(0, int(cx - r)), min(nx, int(cx + r) + 1)
        if z0 >= z1 or y0 >= y1 or x0 >= x1:
            continue
        d = ((zz[z0:z1, None, None] - cz) ** 2 + (yy[None, y0:y1, None] - cy) ** 2 +
             (xx[None, None, x0:x1] - cx) ** 2)
        mask[z0:z1, y0:y1, x0:x1] |= d <= r * r
    return mask.to(torch.uint8)


def batch_shapes(n: int = 64, seed: int = 0):
    """Per-axis dims drawn from {96, 128, 192, 256, 384, 512}, sigma from {2, 4, 8},
    foreground from U(5%, 30%): the batched workload's volumes."""
    g = np.random.default_rng(seed)
    dims = [96, 128, 192, 256, 384, 512]
    out = []
    for _ in range(n):
        shape = tuple(int(v) for v in g.choice(dims, size=3))
        out.append((shape, float(g.choice([2.0, 4.0, 8.0])), float(g.uniform(0.05, 0.30))))
    return out
