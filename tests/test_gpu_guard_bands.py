"""Out-of-bounds checks by guard bands (run with -m gpu).

compute-sanitizer is not available where these tests run, so every device
buffer a kernel touches is placed inside a larger allocation whose 4 KiB on
either side hold a sentinel byte pattern:

  * outputs, field outputs, bins and caller workspaces: after the call the
    guards must still hold the sentinel (no write past either end);
  * inputs: the guards hold a pattern that would change the result if read
    (mask bytes 0xFF = set voxels; uint16 values 0xA5A5), and the result must
    equal, bit for bit, the same call on plain buffers (no read past either end
    that reaches the result).

Every entry point that runs kernels on device buffers is covered: the diffusion
forms (FP32, FP64, 16-bit CUDA-core and tensor-core passes, narrow and wide
radius, uint8 and bit-packed masks), the batched plan, bit-packing, morphology,
the field combination, the cylinder mask, the implant masks and both histograms.
The offsets keep each buffer 4 KiB aligned, as a fresh allocation would be.
"""
import numpy as np
import pytest
import torch

from maxibone_b200 import _lib, device, gauss_kernel
from maxibone_b200.fields import combine_fields, mask_cylinder
from maxibone_b200.geometry import compute_front_back_masks
from maxibone_b200.histograms import axis_histograms, field_histogram
from maxibone_b200.morphology import dilate_3d_sphere, dilate_3d_sphere_bitpacked, erode_3d_sphere
from maxibone_b200.synthetic import random_mask, spheres_mask

pytestmark = pytest.mark.gpu

GUARD_BYTES = 4096
OUT_SENTINEL = 0xA5   # outputs: any write into the guard changes it
MASK_SENTINEL = 0xFF  # mask inputs: a read of the guard would add set voxels


class Guarded:
    """A contiguous CUDA tensor `t` of `shape` with GUARD_BYTES of `sentinel`
    bytes before and after it in the same allocation."""

    def __init__(self, shape, dtype, sentinel=OUT_SENTINEL, init=None):
        self.n = int(np.prod(shape))
        self.esz = torch.empty((), dtype=dtype).element_size()
        self.g = GUARD_BYTES // self.esz
        self.sentinel = sentinel
        self.buf = torch.empty(self.n + 2 * self.g, dtype=dtype, device="cuda")
        self.buf.view(torch.uint8).fill_(sentinel)
        self.t = self.buf[self.g:self.g + self.n].view(shape)
        if init is not None:
            self.t.copy_(init)

    def intact(self) -> bool:
        b = self.buf.view(torch.uint8)
        return bool((b[:GUARD_BYTES] == self.sentinel).all()) and bool((b[-GUARD_BYTES:] == self.sentinel).all())


def _bytes_equal(a: torch.Tensor, b: torch.Tensor) -> bool:
    return torch.equal(a.contiguous().view(torch.uint8), b.contiguous().view(torch.uint8))


def _pack(mask: np.ndarray) -> np.ndarray:
    bits = mask.reshape(-1, 32) != 0
    w = (bits.astype(np.uint64) << np.arange(31, -1, -1, dtype=np.uint64)).sum(axis=1)
    return w.astype(np.uint32)


# (field, shape, sigma, mask format, repetitions, tensor cores)
DIFFUSION_CASES = [
    ("f32", (17, 23, 41), 1.5, "u8", 3, True),          # scalar staging paths, ragged tiles
    ("f32", (40, 64, 96), 8.0, "u8", 3, True),          # vector staging paths, radius 32
    ("f32", (33, 40, 64), 3.0, "bitpacked", 3, True),   # bit-packed mask
    ("f64", (20, 30, 40), 2.0, "u8", 2, True),          # FP64 form
    ("bf16", (30, 70, 100), 2.0, "u8", 3, False),       # 16-bit CUDA-core passes, error feedback
    ("bf16", (40, 136, 264), 8.0, "u8", 3, True),       # tensor-core z pass + fused y/x kernel, partial tiles
    ("f16", (24, 130, 200), 3.0, "bitpacked", 3, True), # fused y/x kernel, bit-packed mask, ragged tiles
    ("f16", (24, 160, 200), 10.0, "u8", 2, True),       # tensor-core wide-radius passes (r = 40)
]


@pytest.mark.parametrize("field,shape,sigma,fmt,reps,tc", DIFFUSION_CASES)
def test_diffusion_stays_inside_its_buffers(field, shape, sigma, fmt, reps, tc):
    mask = spheres_mask(shape, 8, (2, 7), seed=sum(shape))
    mask[random_mask(shape, 0.01, seed=3) > 0] = 1
    kernel = gauss_kernel(sigma).astype(np.float32)
    fo_dtype = torch.float64 if field == "f64" else torch.float32
    n = int(np.prod(shape))
    if fmt == "u8":
        host_mask = torch.from_numpy(mask)
    else:
        host_mask = torch.from_numpy(_pack(mask).view(np.int32))
    opts = dict(field=field, tensor_cores=tc, shape=shape if fmt == "bitpacked" else None)

    plain_out = torch.empty(shape, dtype=torch.uint16, device="cuda")
    plain_field = torch.empty(shape, dtype=fo_dtype, device="cuda")
    device.diffuse(host_mask.cuda(), kernel, reps, output=plain_out, field_out=plain_field, **opts)

    gm = Guarded(tuple(host_mask.shape), host_mask.dtype, MASK_SENTINEL, init=host_mask.cuda())
    go = Guarded(shape, torch.uint16)
    gf = Guarded(shape, fo_dtype)
    gw = Guarded((device.workspace_bytes(shape, field),), torch.uint8)
    device.diffuse(gm.t, kernel, reps, output=go.t, field_out=gf.t, workspace=gw.t, **opts)
    torch.cuda.synchronize()
    device.tensor_core_status()

    assert go.intact() and gf.intact() and gw.intact(), "write outside an output or the workspace"
    assert _bytes_equal(go.t, plain_out), "uint16 output differs from the plain-buffer run"
    assert _bytes_equal(gf.t, plain_field), "field output differs from the plain-buffer run"
    assert n == plain_out.numel()


def test_batch_plan_stays_inside_its_buffers():
    shapes = [(40, 72, 136), (24, 100, 90), (56, 64, 64)]
    sigmas = [2.0, 4.0, 8.0]
    masks = [spheres_mask(s, 6, (2, 6), seed=i + 50) for i, s in enumerate(shapes)]
    kernels = [gauss_kernel(s).astype(np.float32) for s in sigmas]
    reps = 3

    def run(mask_ts, outs, fos):
        plan = device.BatchPlan(mask_ts, kernels, reps, outputs=outs, field="bf16", field_outs=fos)
        plan.run()
        torch.cuda.synchronize()
        plan.close()
        device.tensor_core_status()

    plain_outs = [torch.empty(s, dtype=torch.uint16, device="cuda") for s in shapes]
    plain_fos = [torch.empty(s, dtype=torch.float32, device="cuda") for s in shapes]
    run([torch.from_numpy(m).cuda() for m in masks], plain_outs, plain_fos)

    gms = [Guarded(s, torch.uint8, MASK_SENTINEL, init=torch.from_numpy(m).cuda()) for s, m in zip(shapes, masks)]
    gos = [Guarded(s, torch.uint16) for s in shapes]
    gfs = [Guarded(s, torch.float32) for s in shapes]
    run([g.t for g in gms], [g.t for g in gos], [g.t for g in gfs])
    for i in range(len(shapes)):
        assert gos[i].intact() and gfs[i].intact(), f"volume {i}: write outside its buffers"
        assert _bytes_equal(gos[i].t, plain_outs[i]) and _bytes_equal(gfs[i].t, plain_fos[i]), f"volume {i}"


def test_bitpacking_stays_inside_its_buffers():
    n = 32 * 1000
    mask = (np.random.default_rng(4).random(n) > 0.7).astype(np.uint8)
    gm = Guarded((n,), torch.uint8, MASK_SENTINEL, init=torch.from_numpy(mask).cuda())
    gp = Guarded((n // 32,), torch.int32)
    gu = Guarded((n,), torch.uint8)
    st = torch.cuda.current_stream().cuda_stream
    _lib.check(_lib.lib().maxi_bitpack_encode(gm.t.data_ptr(), n, gp.t.data_ptr(), st))
    _lib.check(_lib.lib().maxi_bitpack_decode(gp.t.data_ptr(), n, gu.t.data_ptr(), st))
    torch.cuda.synchronize()
    assert gp.intact() and gu.intact()
    np.testing.assert_array_equal(gp.t.cpu().numpy().view(np.uint32), _pack(mask))
    np.testing.assert_array_equal(gu.t.cpu().numpy(), mask)


def test_morphology_stays_inside_its_buffers():
    shape = (20, 40, 64)
    mask = random_mask(shape, 0.02, seed=11)
    for fn in (dilate_3d_sphere, erode_3d_sphere):
        src = torch.from_numpy(mask if fn is dilate_3d_sphere else 1 - mask).cuda()
        plain = torch.empty_like(src)
        fn(src, 5, plain)
        gm = Guarded(shape, torch.uint8, MASK_SENTINEL, init=src)
        gr = Guarded(shape, torch.uint8)
        fn(gm.t, 5, gr.t)
        torch.cuda.synchronize()
        assert gr.intact() and torch.equal(gr.t, plain), fn.__name__
    words = torch.from_numpy(_pack(mask).view(np.int32).reshape(shape[0], shape[1], shape[2] // 32)).cuda()
    plain = torch.empty_like(words)
    dilate_3d_sphere_bitpacked(words, 5, plain)
    gm = Guarded(tuple(words.shape), torch.int32, MASK_SENTINEL, init=words)
    gr = Guarded(tuple(words.shape), torch.int32)
    dilate_3d_sphere_bitpacked(gm.t, 5, gr.t)
    torch.cuda.synchronize()
    assert gr.intact() and torch.equal(gr.t, plain)


def test_field_steps_stay_inside_their_buffers():
    shape = (12, 64, 64)
    rng = np.random.default_rng(6)
    gauss = torch.from_numpy(rng.integers(0, 40000, shape, dtype=np.uint16).view(np.int16)).cuda()
    edt = torch.from_numpy(rng.integers(0, 40000, shape, dtype=np.uint16).view(np.int16)).cuda()
    plain = combine_fields(gauss, edt)
    gg = Guarded(shape, torch.int16, init=gauss)
    ge = Guarded(shape, torch.int16, init=edt)
    go = Guarded(shape, torch.int16)
    combine_fields(gg.t, ge.t, output=go.t)
    torch.cuda.synchronize()
    assert go.intact() and torch.equal(go.t, plain)

    plain = gauss.clone()
    mask_cylinder(plain)
    gc = Guarded(shape, torch.int16, init=gauss)
    mask_cylinder(gc.t)
    torch.cuda.synchronize()
    assert gc.intact() and torch.equal(gc.t, plain)


def test_implant_masks_stay_inside_their_buffers():
    shape = (16, 40, 48)
    nz, ny, nx = shape
    zz, yy, xx = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    implant = (((yy - ny / 2 - 0.2 * zz) ** 2 + (xx - nx / 2) ** 2) < 8 ** 2).astype(np.uint8)
    rng = np.random.default_rng(7)
    E = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    UVWp = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    cm = np.array(np.nonzero(implant)).mean(axis=1)
    cp = rng.normal(size=3)
    src = torch.from_numpy(implant).cuda()
    plain = [torch.empty_like(src) for _ in range(4)]
    compute_front_back_masks(src, 1.5, E, cm, cp, UVWp, *plain)
    gm = Guarded(shape, torch.uint8, MASK_SENTINEL, init=src)
    gouts = [Guarded(shape, torch.uint8) for _ in range(4)]
    compute_front_back_masks(gm.t, 1.5, E, cm, cp, UVWp, *[g.t for g in gouts])
    torch.cuda.synchronize()
    for g, p in zip(gouts, plain):
        assert g.intact() and torch.equal(g.t, p)


def test_histograms_stay_inside_their_buffers():
    rng = np.random.default_rng(8)
    vshape, fshape = (8, 48, 40), (4, 24, 20)
    voxels = torch.from_numpy(rng.integers(0, 65536, vshape, dtype=np.uint16).view(np.int16)).cuda()
    field = torch.from_numpy(rng.integers(0, 65536, fshape, dtype=np.uint16).view(np.int16)).cuda()
    plain = torch.zeros((32, 64), dtype=torch.int64, device="cuda")
    field_histogram(voxels, field, (0, 1, 2), plain, (1, 65535), (1, 65535), 0)
    gv = Guarded(vshape, torch.int16, init=voxels)
    gf = Guarded(fshape, torch.int16, init=field)
    gb = Guarded((32, 64), torch.int64, init=torch.zeros((32, 64), dtype=torch.int64, device="cuda"))
    field_histogram(gv.t, gf.t, (0, 1, 2), gb.t, (1, 65535), (1, 65535), 0)
    torch.cuda.synchronize()
    assert gb.intact() and torch.equal(gb.t, plain)

    gshape, vb, center = (8, 48, 40), 64, (24, 20)
    n_r = 32
    dims = (gshape[2], gshape[1], gshape[0], n_r)
    plain = [torch.zeros((d, vb), dtype=torch.int64, device="cuda") for d in dims]
    axis_histograms(voxels, (0, 0, 0), *plain, center, (1, 65535), 0)
    gbins = [Guarded((d, vb), torch.int64, init=torch.zeros((d, vb), dtype=torch.int64, device="cuda"))
             for d in dims]
    axis_histograms(gv.t, (0, 0, 0), *[g.t for g in gbins], center, (1, 65535), 0)
    torch.cuda.synchronize()
    for g, p, name in zip(gbins, plain, "xyzr"):
        assert g.intact() and torch.equal(g.t, p), name


def test_guard_helper_detects_a_write_into_the_guard():
    """The check itself: a byte written just past the end is seen (a host-side copy, no kernel of ours)."""
    g = Guarded((100,), torch.float32)
    assert g.intact()
    g.buf[g.g + g.n] = 0.0
    assert not g.intact()
    g2 = Guarded((100,), torch.float32)
    g2.buf[g2.g - 1] = 0.0
    assert not g2.intact()
