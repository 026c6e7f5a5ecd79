// 3-D sphere dilation and erosion of masks: the reference's morphology module
// (src/lib/cpp/gpu/morphology.cc, cpu_seq/morphology.cc; bound by
// src/pybind/morphology-pybind.cc:24-76,147-150), the step that prepares the
// implant mask before the diffusion (src/processing_steps/0750_bone_region.py:162 via
// src/lib/py/helpers.py:326-349 and morph_3d, :805-850).
//
// uint8 form: result[z,y,x] = 1 iff, over every in-volume offset with
// pz^2 + py^2 + px^2 <= r^2, some voxel is nonzero (dilation) / every voxel has bit 0
// set (erosion: std::bit_and of a bool and a byte).  Offsets outside the volume
// take no part.
//
// Bit-packed form: uint32 words, MSB first along x.  The reference builds one 32-bit
// kernel row per (pz, py) holding x offsets -r .. 31 - r, and reads the three words
// around each output word; with the GPU build's shifts (a shift by 32 or more, or by a
// negative amount, gives 0) that is the sphere with x offsets clipped at 31 - r.
//
// Three passes over packed words, radius <= 32:
//   1. x-runs: X_w[z][y][i] = OP over x offsets -w .. min(w, P) of the row (P = r for
//      the uint8 form, 31 - r for the bit-packed one), w = 0 .. r, built incrementally
//      with one funnel shift each way per step from the word and its two neighbours.
//   2. discs: D_k[z][y][i] = OP over in-volume py of X_{isqrt(r^2 - k^2 - py^2)}[z][y+py][i]
//      for k = 0 .. r (the sphere's cross-section at |pz| = k).
//   3. z: out[z][y][i] = OP over in-volume pz of D_{|pz|}[z+pz][y][i].
// OP is OR for dilation and AND for erosion; outside-volume words and the padding bits
// of a row are the neutral element.  Each output word costs about (pi/2) r^2 + 3r reads
// instead of the (2r+1)^2 * 32 bit steps of the direct form.
#include <vector>

#include "common.cuh"
#include "host_util.h"

namespace maxi {
namespace {

constexpr int kMorphMaxRadius = 32;

template <bool DILATE>
__device__ __forceinline__ uint32_t op(uint32_t a, uint32_t b) {
    return DILATE ? (a | b) : (a & b);
}

__device__ __forceinline__ int isqrt_small(int n) {  // floor(sqrt(n)), 0 <= n <= 2 * 32^2
    int r = (int) sqrtf((float) n);
    while (r * r > n) r--;
    while ((r + 1) * (r + 1) <= n) r++;
    return r;
}

// Pass 1.  Word i of a row; its bits at x offset d come from the 96-bit stream
// (left, word, right): d < 0 from funnelshift_rc(word, left, -d), d > 0 from
// funnelshift_lc(right, word, d).
template <bool DILATE>
__global__ void morph_xruns(const uint32_t *__restrict__ in, uint32_t *__restrict__ xr, int64_t words, int nw,
                            int radius, int pmax) {
    const uint32_t neutral = DILATE ? 0u : 0xffffffffu;
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int i = (int) (idx % nw);
        const uint32_t mid = __ldg(in + idx);
        const uint32_t left = i > 0 ? __ldg(in + idx - 1) : neutral;
        const uint32_t right = i < nw - 1 ? __ldg(in + idx + 1) : neutral;
        uint32_t acc = neutral;
        for (int w = 0; w <= radius; w++) {
            if (-w <= pmax) acc = op<DILATE>(acc, w == 0 ? mid : __funnelshift_rc(mid, left, w));
            if (w > 0 && w <= pmax) acc = op<DILATE>(acc, __funnelshift_lc(right, mid, w));
            xr[(int64_t) w * words + idx] = acc;
        }
    }
}

// Pass 2.  One thread per word (lanes along x); all disc radii for that word.
template <bool DILATE>
__global__ void morph_discs(const uint32_t *__restrict__ xr, uint32_t *__restrict__ disc, int64_t words, int ny,
                            int nw, int radius) {
    const uint32_t neutral = DILATE ? 0u : 0xffffffffu;
    const int64_t plane = (int64_t) ny * nw;
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int y = (int) ((idx % plane) / nw);
        for (int k = 0; k <= radius; k++) {
            const int r2 = radius * radius - k * k;
            const int h = isqrt_small(r2);
            const int lo = max(-h, -y), hi = min(h, ny - 1 - y);
            uint32_t acc = neutral;
            for (int py = lo; py <= hi; py++) {
                const int w = isqrt_small(r2 - py * py);
                acc = op<DILATE>(acc, __ldg(xr + (int64_t) w * words + idx + (int64_t) py * nw));
            }
            disc[(int64_t) k * words + idx] = acc;
        }
    }
}

// Pass 3.
template <bool DILATE>
__global__ void morph_z(const uint32_t *__restrict__ disc, uint32_t *__restrict__ out, int64_t words, int nz,
                        int64_t plane, int radius) {
    const uint32_t neutral = DILATE ? 0u : 0xffffffffu;
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int z = (int) (idx / plane);
        const int lo = max(-radius, -z), hi = min(radius, nz - 1 - z);
        uint32_t acc = neutral;
        for (int pz = lo; pz <= hi; pz++)
            acc = op<DILATE>(acc, __ldg(disc + (int64_t) abs(pz) * words + idx + (int64_t) pz * plane));
        out[idx] = acc;
    }
}

// uint8 rows -> packed words (MSB first), padding bits neutral.  One thread per word.
template <bool DILATE>
__global__ void morph_pack(const uint8_t *__restrict__ in, uint32_t *__restrict__ packed, int64_t words, int nx,
                           int nw) {
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const int64_t row = idx / nw;
        const int x0 = (int) (idx - row * nw) * 32;
        const uint8_t *p = in + row * nx;
        uint32_t w = 0;
        for (int b = 0; b < 32; b++) {
            const int x = x0 + b;
            const uint32_t bit = x < nx ? (DILATE ? (p[x] != 0) : (p[x] & 1)) : (DILATE ? 0u : 1u);
            w |= bit << (31 - b);
        }
        packed[idx] = w;
    }
}

// Packed words -> uint8 0/1 voxels.  One thread per voxel.
__global__ void morph_unpack(const uint32_t *__restrict__ packed, uint8_t *__restrict__ out, int64_t voxels, int nx,
                             int nw) {
    for (int64_t v = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; v < voxels;
         v += (int64_t) gridDim.x * blockDim.x) {
        const int64_t row = v / nx;
        const int x = (int) (v - row * nx);
        out[v] = (uint8_t) ((__ldg(packed + row * nw + (x >> 5)) >> (31 - (x & 31))) & 1u);
    }
}

unsigned grid_for(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned) std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t) sms * 16));
}

// The three passes from `in` to `out` (both packed, words = nz * ny * nw) with the
// x offsets clipped at pmax; scratch holds 2 * (radius + 1) * words words.
template <bool DILATE>
void morph_passes(const uint32_t *in, uint32_t *out, uint32_t *scratch, int64_t nz, int64_t ny, int64_t nw,
                  int radius, int pmax, cudaStream_t st) {
    const int64_t words = nz * ny * nw;
    uint32_t *xr = scratch, *disc = scratch + (int64_t) (radius + 1) * words;
    const unsigned g = grid_for(words);
    morph_xruns<DILATE><<<g, 256, 0, st>>>(in, xr, words, (int) nw, radius, pmax);
    morph_discs<DILATE><<<g, 256, 0, st>>>(xr, disc, words, (int) ny, (int) nw, radius);
    morph_z<DILATE><<<g, 256, 0, st>>>(disc, out, words, (int) nz, ny * nw, radius);
}

int check_shape(int64_t nz, int64_t ny, int64_t n_inner, int64_t radius) {
    if (nz <= 0 || ny <= 0 || n_inner <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "shape (%lld, %lld, %lld) has an empty axis", (long long) nz,
                         (long long) ny, (long long) n_inner);
    if (radius < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "negative radius");
    if (radius > kMorphMaxRadius)
        return set_error(MAXI_ERR_UNSUPPORTED, "sphere radius %lld: at most %d per call (apply radius-32 spheres "
                         "repeatedly for larger ones, as the reference's morph_3d does with 16)",
                         (long long) radius, kMorphMaxRadius);
    if (nz >= (int64_t(1) << 31) || ny >= (int64_t(1) << 31) || n_inner >= (int64_t(1) << 31))
        return set_error(MAXI_ERR_UNSUPPORTED, "axes of 2^31 or more are not served");
    return MAXI_OK;
}

int alloc_scratch(uint32_t **p, size_t bytes, cudaStream_t st) {
    if (cudaMallocAsync(reinterpret_cast<void **>(p), bytes, st) != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of morphology scratch", bytes);
    }
    return MAXI_OK;
}

}  // namespace
}  // namespace maxi

using namespace maxi;

extern "C" int maxi_morphology_sphere_bitpacked(const uint32_t *voxels, uint32_t *result, int64_t nz, int64_t ny,
                                                int64_t nw, int64_t radius, int dilate, void *stream) {
    clear_error();
    if (!voxels || !result) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    int rc = check_shape(nz, ny, nw, radius);
    if (rc) return rc;
    if (radius > 31)  // the kernel row would lose offset 0
        return set_error(MAXI_ERR_UNSUPPORTED, "bit-packed sphere radius %lld: at most 31", (long long) radius);
    if ((rc = require_device())) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t words = nz * ny * nw;
    uint32_t *scratch = nullptr;
    if ((rc = alloc_scratch(&scratch, (size_t) 2 * (radius + 1) * words * sizeof(uint32_t), st))) return rc;
    const int r = (int) radius, pmax = 31 - r;
    if (dilate) morph_passes<true>(voxels, result, scratch, nz, ny, nw, r, pmax, st);
    else morph_passes<false>(voxels, result, scratch, nz, ny, nw, r, pmax, st);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "bit-packed sphere morphology");
}

extern "C" int maxi_morphology_sphere(const uint8_t *voxels, uint8_t *result, int64_t nz, int64_t ny, int64_t nx,
                                      int64_t radius, int dilate, void *stream) {
    clear_error();
    if (!voxels || !result) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    int rc = check_shape(nz, ny, nx, radius);
    if (rc) return rc;
    if ((rc = require_device())) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t nw = ceil_div(nx, 32), words = nz * ny * nw;
    uint32_t *scratch = nullptr;
    // packed input, packed result, then the pass scratch
    if ((rc = alloc_scratch(&scratch, (size_t) (2 + 2 * (radius + 1)) * words * sizeof(uint32_t), st))) return rc;
    uint32_t *packed = scratch, *packed_out = scratch + words, *pass = scratch + 2 * words;
    const int r = (int) radius;
    const unsigned g = grid_for(words);
    if (dilate) {
        morph_pack<true><<<g, 256, 0, st>>>(voxels, packed, words, (int) nx, (int) nw);
        morph_passes<true>(packed, packed_out, pass, nz, ny, nw, r, r, st);
    } else {
        morph_pack<false><<<g, 256, 0, st>>>(voxels, packed, words, (int) nx, (int) nw);
        morph_passes<false>(packed, packed_out, pass, nz, ny, nw, r, r, st);
    }
    const int64_t voxels_n = nz * ny * nx;
    morph_unpack<<<grid_for(voxels_n), 256, 0, st>>>(packed_out, result, voxels_n, (int) nx, (int) nw);
    cudaError_t e = cudaGetLastError();
    cudaFreeAsync(scratch, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "sphere morphology");
}
