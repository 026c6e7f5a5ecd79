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
// Two kernels over packed words, radius <= 32:
//   1. morph_plane_discs, one block per tile of a plane (16 rows, up to 32 words):
//      the tile's rows +- r with one halo word each side go to shared memory; there
//      the x-runs X_w = OP over x offsets -w .. min(w, P) (P = r for the uint8 form,
//      31 - r for the bit-packed one), w = 0 .. r, are built incrementally with one
//      funnel shift each way per step; then each output word gets the discs
//      D_k = OP over py of X_{isqrt(r^2 - k^2 - py^2)}[y + py], k = 0 .. r (the
//      sphere's cross-section at |pz| = k), written to global scratch.
//   2. morph_z: out[z][y][i] = OP over in-volume pz of D_{|pz|}[z+pz][y][i].
// OP is OR for dilation and AND for erosion; outside-volume rows and words and the
// padding bits of a row are the neutral element.  Each output word costs about
// (pi/2) r^2 shared-memory reads and 3r global accesses, instead of the
// (2r+1)^2 * 32 bit steps of the direct form.
#include <map>
#include <mutex>
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

constexpr int kTileRows = 16;

struct PlaneTile {
    int nw, ny, radius, pmax, tile_words;  // tile_words: words per tile along x (<= 32)
    int64_t x_tiles, y_tiles, tiles;
};

size_t plane_tile_smem(int radius, int tile_words) {
    const int rows = kTileRows + 2 * radius;
    return (size_t) rows * (tile_words + 2) * 4 + (size_t) (radius + 1) * rows * tile_words * 4 +
           (size_t) (radius + 1) * (2 * radius + 1);
}

// Pass 1 (x-runs and discs).  Block: 32 lanes along x by 8 warps along y.  Bits at x
// offset d of word j come from the stream (left, word, right): d < 0 from
// funnelshift_rc(word, left, -d), d > 0 from funnelshift_lc(right, word, d).
template <bool DILATE>
__global__ void __launch_bounds__(256) morph_plane_discs(const uint32_t *__restrict__ in, uint32_t *__restrict__ disc,
                                                         int64_t words, PlaneTile t) {
    const uint32_t neutral = DILATE ? 0u : 0xffffffffu;
    const int r = t.radius, rows = kTileRows + 2 * r, tw = t.tile_words, hw = tw + 2;
    extern __shared__ uint32_t sh[];
    uint32_t *in_s = sh;                                   // [rows][tw + 2]
    uint32_t *xr_s = in_s + rows * hw;                     // [r + 1][rows][tw]
    uint8_t *wtab = reinterpret_cast<uint8_t *>(xr_s + (r + 1) * rows * tw);  // [r + 1][2r + 1]
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (r + 1) * (2 * r + 1); i += blockDim.x) {
        const int k = i / (2 * r + 1), py = i % (2 * r + 1) - r;
        const int n = r * r - k * k - py * py;
        wtab[i] = (uint8_t) (n < 0 ? 0xff : isqrt_small(n));
    }
    const int64_t plane = (int64_t) t.ny * t.nw;
    for (int64_t tile = blockIdx.x; tile < t.tiles; tile += gridDim.x) {
        const int64_t xt = tile % t.x_tiles, rest = tile / t.x_tiles;
        const int64_t yt = rest % t.y_tiles, z = rest / t.y_tiles;
        const int x0 = (int) xt * tw, y0 = (int) yt * kTileRows;
        const uint32_t *pl = in + z * plane;
        __syncthreads();  // the previous tile is done with the shared arrays
        for (int i = threadIdx.x; i < rows * hw; i += blockDim.x) {
            const int row = i / hw, c = i % hw;
            const int y = y0 - r + row, x = x0 - 1 + c;
            in_s[i] = (y >= 0 && y < t.ny && x >= 0 && x < t.nw) ? __ldg(pl + (int64_t) y * t.nw + x) : neutral;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < rows * tw; i += blockDim.x) {
            const int row = i / tw, j = i % tw;
            const int y = y0 - r + row;
            const bool inside = y >= 0 && y < t.ny && x0 + j < t.nw;
            const uint32_t left = in_s[row * hw + j], mid = in_s[row * hw + j + 1], right = in_s[row * hw + j + 2];
            uint32_t acc = neutral;
            for (int w = 0; w <= r; w++) {
                if (inside) {
                    if (-w <= t.pmax) acc = op<DILATE>(acc, w == 0 ? mid : __funnelshift_rc(mid, left, w));
                    if (w > 0 && w <= t.pmax) acc = op<DILATE>(acc, __funnelshift_lc(right, mid, w));
                }
                xr_s[(w * rows + row) * tw + j] = acc;
            }
        }
        __syncthreads();
        // Each warp writes rows `warp` and `warp + 8` of the tile (8 warps, 16 rows), the
        // two dependency chains sharing the table lookups.
        if (lane < tw && x0 + lane < t.nw && y0 + warp < t.ny) {
            const bool second = y0 + warp + 8 < t.ny;
            const int stride = rows * tw;
            const uint32_t *c0 = xr_s + (warp + r) * tw + lane, *c1 = c0 + 8 * tw;  // row y of X_0
            uint32_t *d0 = disc + z * plane + (int64_t) (y0 + warp) * t.nw + x0 + lane;
            uint32_t *d1 = d0 + (int64_t) 8 * t.nw;
            for (int k = 0; k <= r; k++) {
                // rows y +- py of X_w with w = isqrt(r^2 - k^2 - py^2), py = 0 .. isqrt(r^2 - k^2)
                const uint8_t *wk = wtab + k * (2 * r + 1) + r;
                uint32_t a0 = c0[wk[0] * stride], a1 = c1[wk[0] * stride];
                for (int py = 1; py <= r && wk[py] != 0xff; py++) {
                    const int o = wk[py] * stride, d = py * tw;
                    a0 = op<DILATE>(a0, op<DILATE>(c0[o + d], c0[o - d]));
                    a1 = op<DILATE>(a1, op<DILATE>(c1[o + d], c1[o - d]));
                }
                d0[(int64_t) k * words] = a0;
                if (second) d1[(int64_t) k * words] = a1;
            }
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

// uint8 rows -> packed words (MSB first), padding bits neutral.  One thread per word;
// VEC: rows are whole words (nx % 32 == 0) and 16-byte aligned, two 16-byte loads.
template <bool DILATE, bool VEC>
__global__ void morph_pack(const uint8_t *__restrict__ in, uint32_t *__restrict__ packed, int64_t words, int nx,
                           int nw) {
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (int64_t) gridDim.x * blockDim.x) {
        uint32_t w = 0;
        if (VEC) {
            const uint4 *p = reinterpret_cast<const uint4 *>(in + idx * 32);
            const uint4 q0 = __ldcs(p), q1 = __ldcs(p + 1);
            const uint32_t u[8] = {q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, q1.z, q1.w};
#pragma unroll
            for (int b = 0; b < 32; b++) {
                const uint32_t byte = (u[b >> 2] >> (8 * (b & 3))) & 0xffu;
                w |= (DILATE ? (uint32_t) (byte != 0) : (byte & 1u)) << (31 - b);
            }
        } else {
            const int64_t row = idx / nw;
            const int x0 = (int) (idx - row * nw) * 32;
            const uint8_t *p = in + row * nx;
            for (int b = 0; b < 32; b++) {
                const int x = x0 + b;
                const uint32_t bit = x < nx ? (DILATE ? (p[x] != 0) : (p[x] & 1)) : (DILATE ? 0u : 1u);
                w |= bit << (31 - b);
            }
        }
        packed[idx] = w;
    }
}

// Packed words -> uint8 0/1 voxels.  One thread per word; VEC as for morph_pack.
template <bool VEC>
__global__ void morph_unpack(const uint32_t *__restrict__ packed, uint8_t *__restrict__ out, int64_t words, int nx,
                             int nw) {
    for (int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; idx < words;
         idx += (int64_t) gridDim.x * blockDim.x) {
        const uint32_t w = __ldg(packed + idx);
        if (VEC) {
            uint32_t u[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
            for (int b = 0; b < 32; b++) u[b >> 2] |= ((w >> (31 - b)) & 1u) << (8 * (b & 3));
            uint4 *p = reinterpret_cast<uint4 *>(out + idx * 32);
            __stcs(p, make_uint4(u[0], u[1], u[2], u[3]));
            __stcs(p + 1, make_uint4(u[4], u[5], u[6], u[7]));
        } else {
            const int64_t row = idx / nw;
            const int x0 = (int) (idx - row * nw) * 32;
            uint8_t *p = out + row * nx;
            for (int b = 0; b < 32 && x0 + b < nx; b++) p[x0 + b] = (uint8_t) ((w >> (31 - b)) & 1u);
        }
    }
}

unsigned grid_for(int64_t n) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return (unsigned) std::max<int64_t>(1, std::min<int64_t>(ceil_div(n, 256), (int64_t) sms * 16));
}

// The passes from `in` to `out` (both packed, words = nz * ny * nw) with the x offsets
// clipped at pmax; scratch holds (radius + 1) * words words.
template <bool DILATE>
int morph_passes(const uint32_t *in, uint32_t *out, uint32_t *scratch, int64_t nz, int64_t ny, int64_t nw,
                 int radius, int pmax, cudaStream_t st) {
    const int64_t words = nz * ny * nw;
    PlaneTile t{};
    t.nw = (int) nw;
    t.ny = (int) ny;
    t.radius = radius;
    t.pmax = pmax;
    t.tile_words = 32;
    while (t.tile_words > 8 && plane_tile_smem(radius, t.tile_words) > 200 * 1024) t.tile_words /= 2;
    t.x_tiles = ceil_div(nw, t.tile_words);
    t.y_tiles = ceil_div(ny, kTileRows);
    t.tiles = t.x_tiles * t.y_tiles * nz;
    const size_t smem = plane_tile_smem(radius, t.tile_words);
    cudaError_t e = cudaFuncSetAttribute(morph_plane_discs<DILATE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int) smem);
    if (e != cudaSuccess) return set_cuda_error(e, "morphology set-up");
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned g1 = (unsigned) std::min<int64_t>(t.tiles, (int64_t) sms * 8);
    morph_plane_discs<DILATE><<<g1, 256, smem, st>>>(in, scratch, words, t);
    morph_z<DILATE><<<grid_for(words), 256, 0, st>>>(scratch, out, words, (int) nz, ny * nw, radius);
    return MAXI_OK;
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

// Scratch kept between calls, one grow-only buffer per device: the pipeline applies
// radius-16 spheres over and over, and mapping gigabytes afresh for each call would
// cost more than the passes.  A call holds its device's buffer until it returns.
struct Scratch {
    std::mutex mu;
    uint32_t *buf = nullptr;
    size_t bytes = 0;
};
std::mutex g_scratch_mu;
std::map<int, Scratch *> g_scratch;

// Locks and returns the device's scratch, grown to `bytes`.
int acquire_scratch(size_t bytes, std::unique_lock<std::mutex> &lock, uint32_t **p) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    Scratch *s;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        Scratch *&slot = g_scratch[dev];
        if (!slot) slot = new Scratch();
        s = slot;
    }
    lock = std::unique_lock<std::mutex>(s->mu);
    if (s->bytes < bytes) {
        if (s->buf) {
            cudaDeviceSynchronize();  // earlier calls' work on the old buffer
            cudaFree(s->buf);
            s->buf = nullptr;
            s->bytes = 0;
        }
        if (cudaMalloc(reinterpret_cast<void **>(&s->buf), bytes) != cudaSuccess) {
            cudaGetLastError();
            s->buf = nullptr;
            return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of morphology scratch", bytes);
        }
        s->bytes = bytes;
    }
    *p = s->buf;
    return MAXI_OK;
}

}  // namespace

void release_morphology_scratch() {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    for (auto &kv : g_scratch) {
        std::lock_guard<std::mutex> lk2(kv.second->mu);
        if (kv.second->buf) {
            cudaDeviceSynchronize();
            cudaFree(kv.second->buf);
            kv.second->buf = nullptr;
            kv.second->bytes = 0;
        }
    }
}

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
    std::unique_lock<std::mutex> hold;
    if ((rc = acquire_scratch((size_t) (radius + 1) * words * sizeof(uint32_t), hold, &scratch))) return rc;
    const int r = (int) radius, pmax = 31 - r;
    rc = dilate ? morph_passes<true>(voxels, result, scratch, nz, ny, nw, r, pmax, st)
                : morph_passes<false>(voxels, result, scratch, nz, ny, nw, r, pmax, st);
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaStreamSynchronize(st);  // the scratch is free for the next call
    if (rc) return rc;
    if (e == cudaSuccess) e = e2;
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
    std::unique_lock<std::mutex> hold;
    // packed input, packed result, then the pass scratch
    if ((rc = acquire_scratch((size_t) (2 + (radius + 1)) * words * sizeof(uint32_t), hold, &scratch))) return rc;
    uint32_t *packed = scratch, *packed_out = scratch + words, *pass = scratch + 2 * words;
    const int r = (int) radius;
    const unsigned g = grid_for(words);
    const bool vec = nx % 32 == 0 && ((reinterpret_cast<uintptr_t>(voxels) | reinterpret_cast<uintptr_t>(result)) & 15) == 0;
    if (dilate) {
        if (vec) morph_pack<true, true><<<g, 256, 0, st>>>(voxels, packed, words, (int) nx, (int) nw);
        else morph_pack<true, false><<<g, 256, 0, st>>>(voxels, packed, words, (int) nx, (int) nw);
        rc = morph_passes<true>(packed, packed_out, pass, nz, ny, nw, r, r, st);
    } else {
        if (vec) morph_pack<false, true><<<g, 256, 0, st>>>(voxels, packed, words, (int) nx, (int) nw);
        else morph_pack<false, false><<<g, 256, 0, st>>>(voxels, packed, words, (int) nx, (int) nw);
        rc = morph_passes<false>(packed, packed_out, pass, nz, ny, nw, r, r, st);
    }
    if (rc) {
        cudaStreamSynchronize(st);
        return rc;
    }
    if (vec) morph_unpack<true><<<g, 256, 0, st>>>(packed_out, result, words, (int) nx, (int) nw);
    else morph_unpack<false><<<g, 256, 0, st>>>(packed_out, result, words, (int) nx, (int) nw);
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaStreamSynchronize(st);  // the scratch is free for the next call
    if (e == cudaSuccess) e = e2;
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "sphere morphology");
}
