"""Test oracle for the mask-diffusion path (test infrastructure only).

Only the tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import this package, and only to check results or as the timed CPU
baseline.  The product (``maxibone_b200``) never imports it.

The oracles:

* ``diffusion_in_memory``: ctypes binding of ``diffusion_oracle.c``, a C
  restatement of the reference OpenMP backend
  (src/lib/cpp/cpu/diffusion.cc:31-57,191-195,243-247,295-302,314-320,339-374).
  It is bit-identical to the reference's own module (pinned by the golden
  vectors in tests/golden and, where the reference tree is present, by running
  the reference module built into ``oracle/_ref``).
* ``scipy_chain``: the oracle of the reference's own unit test,
  src/test/test_diffusion.py:49-59 (scipy ``convolve1d`` with mode='constant').
* ``diffusion_f64``: the same algorithm in FP64, the error reference for the
  reduced-precision field forms.

* ``combine_fields``: the numpy Gaussian + EDT field combination of the
  reference's step src/processing_steps/0975_combine_fields.py:38-62, with its
  ``to_int`` restated as ``normalized_convert_u16`` (pinned to the reference's
  compiled ``general.normalized_convert`` by tests/golden).

* ``morphology_sphere`` and ``morphology_sphere_bitpacked``: the reference's 3-D
  sphere dilation / erosion on uint8 and bit-packed masks
  (src/lib/cpp/cpu_seq/morphology.cc, gpu/morphology.cc) in numpy, pinned to the
  compiled module by tests/golden.

* ``implant_masks``: the front / back / implant-shell / solid-implant masks of the
  reference's geometry module (src/lib/cpp/cpu_seq/geometry.cc:112-215) in numpy
  float32, pinned to the compiled module by tests/golden.

* ``field_histogram`` and ``axis_histograms``: the 2-D (field, voxel) and the
  per-axis / radial histograms of the reference's histograms module
  (src/lib/cpp/cpu/histograms.cc:231-305 and :14-80) in numpy, pinned to the
  compiled module by tests/golden.

``reference_module()`` imports the reference's own ``diffusion`` (and
``bitpacking``, ``general``, ``histograms``, ``morphology``, ``geometry``) pybind modules from ``oracle/_ref`` when they have
been built (``make -C oracle ref``).
"""
from __future__ import annotations

import ctypes
import importlib.util
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> None:
    """Compile the C restatement (and the reference modules where the reference tree exists)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref_src = os.environ.get("MAXI_REFERENCE_SRC", "/root/reference/src")
    if os.path.isdir(ref_src):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref_src}"], check=True)


def _lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle_diffusion.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
        lib = ctypes.CDLL(path)
        i64, p = ctypes.c_int64, ctypes.c_void_p
        lib.oracle_diffusion_in_memory.argtypes = [p, i64, i64, i64, p, i64, i64, p, p]
        lib.oracle_diffusion_in_memory.restype = ctypes.c_int
        lib.oracle_diffusion_f64.argtypes = [p, i64, i64, i64, p, i64, i64, p]
        lib.oracle_diffusion_f64.restype = ctypes.c_int
        lib.oracle_diffusion_on_disk_semantics.argtypes = [p, i64, i64, i64, p, i64, i64, p]
        lib.oracle_diffusion_on_disk_semantics.restype = ctypes.c_int
        lib.oracle_diffusion_on_disk_field.argtypes = [p, i64, i64, i64, p, i64, i64, p]
        lib.oracle_diffusion_on_disk_field.restype = ctypes.c_int
        lib.oracle_diffusion_from_field.argtypes = [p, p, i64, i64, i64, p, i64, i64, p]
        lib.oracle_diffusion_from_field.restype = ctypes.c_int
        lib.oracle_f32_to_u8.argtypes = [p, p, i64]
        lib.oracle_f32_to_u8.restype = None
        lib.oracle_convolve_axis_f32.argtypes = [p, p, p, i64, i64, i64, ctypes.c_int, i64]
        lib.oracle_convolve_axis_f32.restype = None
        lib.oracle_bitpack_encode_u32.argtypes = [p, i64, p]
        lib.oracle_bitpack_encode_u32.restype = None
        lib.oracle_bitpack_decode_u32.argtypes = [p, i64, p]
        lib.oracle_bitpack_decode_u32.restype = None
        _LIB = lib
    return _LIB


def _ptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)


def diffusion_in_memory(mask: np.ndarray, kernel: np.ndarray, repititions: int):
    """FP32 reference semantics. Returns (uint16 output, float32 final field)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    nz, ny, nx = m.shape
    out = np.empty(m.shape, np.uint16)
    field = np.empty(m.shape, np.float32)
    rc = _lib().oracle_diffusion_in_memory(_ptr(m), nz, ny, nx, _ptr(k), k.shape[0], int(repititions),
                                           _ptr(out), _ptr(field))
    if rc != 0:
        raise MemoryError("oracle could not allocate its working buffers")
    return out, field


def diffusion_f64(mask: np.ndarray, kernel: np.ndarray, repititions: int) -> np.ndarray:
    """FP64 field after `repititions` steps (kernel promoted to FP64 as given)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    k = np.ascontiguousarray(kernel, dtype=np.float64)
    nz, ny, nx = m.shape
    field = np.empty(m.shape, np.float64)
    rc = _lib().oracle_diffusion_f64(_ptr(m), nz, ny, nx, _ptr(k), k.shape[0], int(repititions), _ptr(field))
    if rc != 0:
        raise MemoryError("oracle could not allocate its working buffers")
    return field


def diffusion_on_disk_semantics(mask: np.ndarray, kernel: np.ndarray, repititions: int) -> np.ndarray:
    """uint16 output of the reference's on-disk variant (mask rebuilt as field == 1.0f each step)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    nz, ny, nx = m.shape
    out = np.empty(m.shape, np.uint16)
    rc = _lib().oracle_diffusion_on_disk_semantics(_ptr(m), nz, ny, nx, _ptr(k), k.shape[0],
                                                   int(repititions), _ptr(out))
    if rc != 0:
        raise MemoryError("oracle could not allocate its working buffers")
    return out


def diffusion_on_disk_u8(mask: np.ndarray, kernel: np.ndarray, repititions: int) -> np.ndarray:
    """uint8 output of the reference CPU backend's on-disk variant: the field of
    the on-disk semantics (mask rebuilt as field == 1.0f each step) converted
    as (uint8) floor(v * 255.0f) (src/lib/cpp/cpu/diffusion.cc:139-144, 459)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    nz, ny, nx = m.shape
    field = np.empty(m.shape, np.float32)
    rc = _lib().oracle_diffusion_on_disk_field(_ptr(m), nz, ny, nx, _ptr(k), k.shape[0], int(repititions),
                                               _ptr(field))
    if rc != 0:
        raise MemoryError("oracle could not allocate its working buffers")
    out = np.empty(m.shape, np.uint8)
    _lib().oracle_f32_to_u8(_ptr(field), _ptr(out), field.size)
    return out


def diffusion_from_field(field: np.ndarray, mask: np.ndarray, kernel: np.ndarray, repititions: int) -> np.ndarray:
    """FP32 field after `repititions` more repetitions from `field` (zero
    boundary at the array's edges): the reference's steps without the initial
    mask -> field conversion (src/lib/cpp/cpu/diffusion.cc:314-320,354-358)."""
    f = np.ascontiguousarray(field, dtype=np.float32)
    m = np.ascontiguousarray(mask, dtype=np.uint8)
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    out = np.empty_like(f)
    nz, ny, nx = f.shape
    rc = _lib().oracle_diffusion_from_field(_ptr(f), _ptr(m), nz, ny, nx, _ptr(k), k.shape[0], int(repititions),
                                            _ptr(out))
    if rc != 0:
        raise MemoryError("oracle could not allocate its working buffers")
    return out


def convolve_axis(field: np.ndarray, kernel: np.ndarray, dim: int) -> np.ndarray:
    """One zero-boundary FP32 pass along axis `dim` (reference diffusion_core)."""
    f = np.ascontiguousarray(field, dtype=np.float32)
    k = np.ascontiguousarray(kernel, dtype=np.float32)
    out = np.empty_like(f)
    nz, ny, nx = f.shape
    _lib().oracle_convolve_axis_f32(_ptr(f), _ptr(k), _ptr(out), nz, ny, nx, int(dim), k.shape[0] // 2)
    return out


def bitpack_encode(mask: np.ndarray) -> np.ndarray:
    """uint8 mask -> uint32 words, MSB first (reference cpu_seq/bitpacking.cc:9-24)."""
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    assert m.size % 32 == 0
    out = np.empty(m.size // 32, np.uint32)
    _lib().oracle_bitpack_encode_u32(_ptr(m), m.size, _ptr(out))
    return out


def bitpack_decode(packed: np.ndarray, n: int) -> np.ndarray:
    p = np.ascontiguousarray(packed, dtype=np.uint32)
    out = np.empty(n, np.uint8)
    _lib().oracle_bitpack_decode_u32(_ptr(p), n, _ptr(out))
    return out


def scipy_chain(mask: np.ndarray, kernel: np.ndarray, repititions: int) -> np.ndarray:
    """The reference unit test's oracle (src/test/test_diffusion.py:49-59), uint16 result."""
    import scipy.ndimage as ndi
    a = np.asarray(mask).astype(bool)
    k = np.asarray(kernel, dtype=np.float32)
    buf0 = a.astype(np.float32)
    buf1 = np.zeros_like(buf0)
    for _ in range(repititions):
        buf1[:] = ndi.convolve1d(buf0, k, axis=0, mode="constant")
        buf0[:] = ndi.convolve1d(buf1, k, axis=1, mode="constant")
        buf1[:] = ndi.convolve1d(buf0, k, axis=2, mode="constant")
        buf1[a] = 1
        buf0, buf1 = buf1, buf0
    return np.floor(buf0 * 65535).astype(np.uint16)


def cylinder_mask(ny: int, nx: int | None = None) -> np.ndarray:
    """bool[ny, nx]: the reference's generate_cylinder_mask (src/lib/py/helpers.py:411-434)."""
    if nx is None:
        nx = ny
    ys = np.linspace(-1, 1, ny)
    xs = np.linspace(-1, 1, nx)
    return (xs[np.newaxis, :] ** 2 + ys[:, np.newaxis] ** 2) < 1


def normalized_convert_u16(x: np.ndarray) -> np.ndarray:
    """normalized_convert<float, uint16_t> (src/lib/cpp/include/general.hh:78-118), the
    3-D path of the reference's to_int (src/lib/py/helpers.py:1013-1038): FP32
    (x - vmin) / (vmax - vmin) * 65535 with vmin, vmax the array's extremes,
    truncated to uint16."""
    x = np.asarray(x, dtype=np.float32)
    vmin, vmax = x.min(), x.max()
    r = (x - vmin) / (vmax - vmin) * np.float32(np.iinfo(np.uint16).max)
    return r.astype(np.uint16)


def combine_fields(gauss: np.ndarray, edt: np.ndarray) -> np.ndarray:
    """The Gaussian + EDT field combination of src/processing_steps/0975_combine_fields.py:38-62
    on uint16 fields [nz, ny, nx] (the cylinder mask spans y and x as
    generate_cylinder_mask(ny, nx); the script passes nx alone, which equals it for
    the square planes it is run on)."""
    nz, ny, nx = edt.shape
    cylinder = cylinder_mask(ny, nx)
    edt_max = edt.max()
    gauss_max = gauss.max()
    combined = gauss.astype(np.float32) / gauss_max
    combined -= edt.astype(np.float32) / edt_max
    combined += np.abs(combined.min())
    combined /= combined.max()
    combined *= cylinder
    combined = normalized_convert_u16(combined)
    combined *= cylinder
    return combined


def field_histogram(voxels: np.ndarray, field: np.ndarray, offset, bins_shape, vrange, frange) -> np.ndarray:
    """uint64[field_bins, voxel_bins]: the reference's field_histogram
    (src/lib/cpp/cpu/histograms.cc:231-305, via src/pybind/histograms-pybind.cc:81-107)
    with the same FP64 expressions: each voxel value inside vrange (others count as 0)
    is binned as floor((voxel_bins - 1) * ((v - vmin) / (vmax - vmin))), the field is
    read at (min(nz - 1, floor(Z * nz/nZ)), floor(Y * ny/nY), floor(X * nx/nX)), zero
    voxels and zero field values are skipped, and rows / columns start at the offset's
    y and x.  Field bins outside [0, field_bins) (undefined in the reference) are skipped."""
    field_bins, voxel_bins = bins_shape
    nZ, nY, nX = voxels.shape
    nz, ny, nx = field.shape
    vmin, vmax = (float(v) for v in vrange)
    fmin, fmax = (float(v) for v in frange)
    _, y_start, x_start = (int(v) for v in offset)
    dz, dy, dx = nz / nZ, ny / nY, nx / nX
    v = voxels.astype(np.float64)
    v = np.where((v >= vmin) & (v <= vmax), v, 0.0)
    vi = np.floor(float(voxel_bins - 1) * ((v - vmin) / (vmax - vmin)))
    z = np.minimum(nz - 1, np.floor(np.arange(nZ) * dz).astype(np.int64))
    y = np.floor(np.arange(nY) * dy).astype(np.int64)
    x = np.floor(np.arange(nX) * dx).astype(np.int64)
    f = field[z[:, None, None], y[None, :, None], x[None, None, :]].astype(np.float64)
    fi = np.floor(float(field_bins - 1) * ((f - fmin) / (fmax - fmin)))
    keep = (v != 0) & (f > 0) & (fi >= 0) & (fi < field_bins)
    keep[:, :y_start, :] = False
    keep[:, :, :x_start] = False
    bins = np.zeros((field_bins, voxel_bins), np.uint64)
    np.add.at(bins, (fi[keep].astype(np.int64), vi[keep].astype(np.int64)), np.uint64(1))
    return bins


def axis_histograms(voxels: np.ndarray, offset, global_shape, voxel_bins: int, n_r: int, center, vrange):
    """(x_bins, y_bins, z_bins, r_bins), uint64 [N, voxel_bins]: the reference's
    axis_histogram (src/lib/cpp/cpu/histograms.cc:14-80, via
    src/pybind/histograms-pybind.cc:30-66).  The block covers global planes
    z_start .. min(z_start + nz_block, Nz) with the global y and x extents; voxels
    at y >= y_start and x >= x_start whose value lies in vrange are binned as
    floor((voxel_bins - 1) * ((v - vmin) / (vmax - vmin))) in FP64 and counted in
    x_bins[x], y_bins[y], z_bins[z] and r_bins[floor(sqrt((x-cx)^2 + (y-cy)^2))].
    Radii at or past n_r (undefined in the reference) are skipped."""
    nz_g, ny_g, nx_g = global_shape
    z_start, y_start, x_start = (int(v) for v in offset)
    cy, cx = (int(c) for c in center)
    vmin, vmax = (float(v) for v in vrange)
    z_end = min(z_start + voxels.shape[0], nz_g)
    blk = voxels[: max(0, z_end - z_start)].reshape(-1, ny_g, nx_g)
    v = blk.astype(np.float64)
    v = np.where((v >= vmin) & (v <= vmax), v, 0.0)
    vi = np.floor(float(voxel_bins - 1) * ((v - vmin) / (vmax - vmin)))
    zz, yy, xx = np.meshgrid(np.arange(z_start, z_end), np.arange(ny_g), np.arange(nx_g), indexing="ij")
    r = np.floor(np.sqrt(((xx - cx) ** 2 + (yy - cy) ** 2).astype(np.float64))).astype(np.int64)
    keep = (v != 0) & (vi < voxel_bins) & (yy >= y_start) & (xx >= x_start)
    out = []
    for coord, n in ((xx, nx_g), (yy, ny_g), (zz, nz_g), (r, n_r)):
        k = keep & (coord < n)
        b = np.zeros((n, voxel_bins), np.uint64)
        np.add.at(b, (coord[k], vi[k].astype(np.int64)), np.uint64(1))
        out.append(b)
    return tuple(out)


def _sphere_offsets(radius: int, px_max: int | None = None):
    r = int(radius)
    out = []
    for pz in range(-r, r + 1):
        for py in range(-r, r + 1):
            w2 = r * r - pz * pz - py * py
            if w2 < 0:
                continue
            w = int(np.floor(np.sqrt(w2)))
            while (w + 1) * (w + 1) <= w2:
                w += 1
            while w * w > w2:
                w -= 1
            hi = w if px_max is None else min(w, px_max)
            if hi >= -w:
                out.append((pz, py, -w, hi))
    return out


def morphology_sphere(mask: np.ndarray, radius: int, dilate: bool, px_max: int | None = None) -> np.ndarray:
    """uint8 0/1 result of the reference's 3-D sphere morphology on a uint8 mask
    (src/lib/cpp/cpu_seq/morphology.cc:14-55, as bound by
    src/pybind/morphology-pybind.cc:24-45,147-149): every in-volume offset with
    pz^2 + py^2 + px^2 <= radius^2 takes part (offsets outside the volume are skipped);
    dilation ORs (v != 0), erosion ANDs (v & 1) -- std::bit_and on a bool and a byte.
    `px_max` clips the x offsets (the bit-packed form's kernel row, below)."""
    m = np.asarray(mask)
    bit = (m != 0) if dilate else ((m & 1) != 0)
    r = int(radius)
    nz, ny, nx = bit.shape
    pad = np.full((nz + 2 * r, ny + 2 * r, nx + 2 * r), not dilate, dtype=bool)
    pad[r:r + nz, r:r + ny, r:r + nx] = bit
    # x-runs: run[w_lo, w_hi][z, y, x] = op over x offsets w_lo..w_hi
    out = np.full(bit.shape, not dilate, dtype=bool)
    cache = {}
    for pz, py, lo, hi in _sphere_offsets(r, px_max):
        key = (lo, hi)
        if key not in cache:
            acc = np.full((nz + 2 * r, ny + 2 * r, nx), not dilate, dtype=bool)
            for px in range(lo, hi + 1):
                sl = pad[:, :, r + px:r + px + nx]
                acc = (acc | sl) if dilate else (acc & sl)
            cache[key] = acc
        sl = cache[key][r + pz:r + pz + nz, r + py:r + py + ny, :]
        out = (out | sl) if dilate else (out & sl)
    return out.astype(np.uint8)


def morphology_sphere_bitpacked(words: np.ndarray, radius: int, dilate: bool) -> np.ndarray:
    """uint32 [nz, ny, nx/32] result of the reference's bit-packed sphere morphology
    (src/lib/cpp/gpu/morphology.cc:103-176 and cpu_seq/morphology.cc:102-176; words
    MSB first along x) with the GPU build's shift semantics, the module the pipeline
    imports (src/lib/py/helpers.py:19): a shift by 32 or more, or by a negative amount,
    gives 0.  Each (pz, py) kernel row holds x offsets -r .. 31 - r only, so the result
    is the uint8 morphology with x offsets clipped at 31 - radius, packed again."""
    w = np.ascontiguousarray(words, dtype=np.uint32)
    bits = np.unpackbits(w.astype(">u4").view(np.uint8), axis=-1).reshape(w.shape[0], w.shape[1], -1)
    res = morphology_sphere(bits, radius, dilate, px_max=31 - int(radius))
    packed = np.packbits(res.astype(np.uint8), axis=-1).view(">u4").astype(np.uint32)
    return packed.reshape(w.shape)


def implant_masks(mask: np.ndarray, voxel_size, E, cm, cp, UVWp, planes=None):
    """(front, back, implant_shell, solid_implant) uint8 masks of the reference's
    compute_front_back_masks (src/lib/cpp/cpu_seq/geometry.cc:112-215, bound by
    src/pybind/geometry-pybind.cc:283-310, called by src/processing_steps/0750_bone_region.py:62),
    in float32 with the reference's operation order (no fused multiply-add, as its
    x86-64 build): uvw = (zyx - cm) @ E, w0 = min(0, min of w over the mask),
    UVW = (uvw - (0, 0, w0)) * voxel_size, (Vp, Wp) from (UVW - cp) @ UVWp,
    r = sqrt(Vp^2 + Wp^2), rmax = per-plane max of r * mask; the comparisons with
    0.7 * rmax are in FP64.  `planes`: evaluate only these z planes (the outputs are
    [len(planes), ny, nx]); w0 still comes from the whole mask."""
    f32 = np.float32
    m = np.asarray(mask)
    E = np.asarray(E, f32).reshape(9)
    cm = np.asarray(cm, f32).reshape(3)
    cp = np.asarray(cp, f32).reshape(3)
    P = np.asarray(UVWp, f32).reshape(9)
    vs = f32(voxel_size)
    nz, ny, nx = m.shape

    def comp(zs, ys, xs, k):
        return (zs * E[k] + ys * E[3 + k]) + xs * E[6 + k]

    w0 = f32(0)
    nzs = np.nonzero(m)
    if nzs[0].size:
        wz = comp(nzs[0].astype(f32) - cm[0], nzs[1].astype(f32) - cm[1], nzs[2].astype(f32) - cm[2], 2)
        w0 = min(f32(0), f32(wz.min()))
    ys = (np.arange(ny, dtype=np.int64).astype(f32) - cm[1])[:, None]
    xs = (np.arange(nx, dtype=np.int64).astype(f32) - cm[2])[None, :]
    zlist = range(nz) if planes is None else list(planes)
    outs = [np.empty((len(zlist), ny, nx), np.uint8) for _ in range(4)]
    for i, z in enumerate(zlist):
        zs = f32(z) - cm[0]
        U = (comp(zs, ys, xs, 0) - f32(0)) * vs
        V = (comp(zs, ys, xs, 1) - f32(0)) * vs
        W = (comp(zs, ys, xs, 2) - f32(w0)) * vs
        a, b, c = U - cp[0], V - cp[1], W - cp[2]
        Vp = (a * P[1] + b * P[4]) + c * P[7]
        Wp = (a * P[2] + b * P[5]) + c * P[8]
        r = np.sqrt(Vp * Vp + Wp * Wp).astype(f32)
        mz = m[z]
        rmax = max(f32(0), f32((r * mz.astype(f32)).max()))
        lim = 0.7 * float(rmax)
        rd = r.astype(np.float64)
        solid = (mz | ((rd < lim) & (W >= 0)).astype(np.uint8)).astype(np.uint8)
        outs[0][i] = ((W > 50) & (solid == 0)).astype(np.uint8)
        outs[1][i] = (W < 0).astype(np.uint8)
        outs[2][i] = (mz & (rd >= lim).astype(np.uint8)).astype(np.uint8)
        outs[3][i] = solid
    return tuple(outs)


def reference_module(name: str = "diffusion"):
    """Import the reference's own CPU pybind module built into oracle/_ref, or None."""
    ref_dir = os.path.join(HERE, "_ref")
    if not os.path.isdir(ref_dir):
        return None
    for f in os.listdir(ref_dir):
        if f.startswith(name + ".") and f.endswith(".so"):
            spec = importlib.util.spec_from_file_location(name, os.path.join(ref_dir, f))
            mod = importlib.util.module_from_spec(spec)
            try:
                spec.loader.exec_module(mod)
            except ImportError:
                return None
            return mod
    return None
