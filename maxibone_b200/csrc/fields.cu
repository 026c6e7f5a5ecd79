// Combination of the Gaussian (diffusion) field with the implant EDT field:
// the step after the diffusion in maxibone's pipeline,
// src/processing_steps/0975_combine_fields.py:38-62.  On uint16 fields G, E
// [nz][ny][nx] and the cylinder mask C[y][x] of generate_cylinder_mask
// (src/lib/py/helpers.py:411-434, here over ny and nx):
//
//   c   = G / max(G) - E / max(E)                     (FP32, as numpy does it)
//   c'  = (c + |min c|) / max(c + |min c|)
//   c'' = c' * C
//   out = to_int(c'') * C,  to_int = normalized_convert<float, uint16_t>
//         (src/lib/cpp/include/general.hh:78-118): (x - vmin) / (vmax - vmin) * 65535, truncated
//
// Every step after c is monotone non-decreasing in c (rounding included), so
// the extremes the later steps need follow from the extremes of c over all
// voxels and over the voxels inside the cylinder: two reduction passes (the
// field maxima, then those extremes) and one conversion pass, each a read of
// both fields -- HBM-bound.  The host does the scalar steps in FP32 between
// the passes.  The cylinder is convex along x for every row, so each row's
// inside voxels are one x interval, found on the host with numpy's own FP64
// arithmetic (linspace(-1, 1, n)[i] = i * (2 / (n - 1)) - 1, last point 1).
#include <cmath>
#include <vector>

#include "common.cuh"
#include "host_util.h"

namespace maxi {
namespace {

struct CombineStats {
    unsigned int gmax, emax;        // field maxima
    unsigned int cmin, cmax;        // extremes of c over all voxels (order-preserving keys)
    unsigned int cmin_in, cmax_in;  // the same inside the cylinder
    unsigned int pad[2];
};

// Float <-> unsigned key with the same order (for atomicMin / atomicMax).
__device__ __forceinline__ unsigned int fkey(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
float key_float(unsigned int k) {
    const unsigned int u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// The voxel loop over the flat volume, 8 voxels per step (16-byte loads) when
// rows allow it, else 1; f(row, x, count) with the step's voxels inside one row.
// f(row, y, x, count).  Chunk and row indices stay below 2^32 (the host checks),
// so the index divisions are 32-bit.
template <typename F>
__device__ __forceinline__ void for_chunks(int64_t rows, int64_t ny, int64_t nx, bool vec, F &&f) {
    const uint32_t step = vec ? 8u : 1u;
    const uint32_t per_row = (uint32_t) (nx / step), yn = (uint32_t) ny;
    const uint32_t total = (uint32_t) (rows * per_row);
    for (uint32_t c = blockIdx.x * blockDim.x + threadIdx.x; c < total; c += gridDim.x * blockDim.x) {
        const uint32_t row = c / per_row;
        const uint32_t y = row % yn;
        f((int64_t) row, (int) y, (int64_t) (c - row * per_row) * step, (int) step);
    }
}

__device__ __forceinline__ void load8(const uint16_t *p, int cnt, float (&v)[8]) {
    if (cnt == 8) {
        const uint4 w = __ldg(reinterpret_cast<const uint4 *>(p));
        const uint32_t a[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int i = 0; i < 4; i++) {
            v[2 * i] = (float) (a[i] & 0xffffu);
            v[2 * i + 1] = (float) (a[i] >> 16);
        }
    } else {
        v[0] = (float) __ldg(p);
    }
}

__device__ __forceinline__ unsigned int warp_max(unsigned int v) { return __reduce_max_sync(0xffffffffu, v); }
__device__ __forceinline__ unsigned int warp_min(unsigned int v) { return __reduce_min_sync(0xffffffffu, v); }

__global__ void field_maxima(const uint16_t *__restrict__ g, const uint16_t *__restrict__ e, int64_t rows, int64_t ny,
                             int64_t nx, bool vec, CombineStats *st) {
    unsigned int gm = 0, em = 0;
    for_chunks(rows, ny, nx, vec, [&](int64_t row, int y, int64_t x, int cnt) {
        float a[8], b[8];
        load8(g + row * nx + x, cnt, a);
        load8(e + row * nx + x, cnt, b);
        for (int i = 0; i < cnt; i++) {
            gm = max(gm, (unsigned int) a[i]);
            em = max(em, (unsigned int) b[i]);
        }
    });
    gm = warp_max(gm);
    em = warp_max(em);
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&st->gmax, gm);
        atomicMax(&st->emax, em);
    }
}

// c = G / gm - E / em with numpy's FP32 operations (no contraction).
__device__ __forceinline__ float combined(float g, float e, float gm, float em) {
    return __fsub_rn(__fdiv_rn(g, gm), __fdiv_rn(e, em));
}

__global__ void combined_extremes(const uint16_t *__restrict__ g, const uint16_t *__restrict__ e, int64_t rows,
                                  int64_t ny, int64_t nx, bool vec, const int2 *__restrict__ inside, float gm, float em,
                                  CombineStats *st) {
    unsigned int lo = 0xffffffffu, hi = 0, lo_in = 0xffffffffu, hi_in = 0;
    for_chunks(rows, ny, nx, vec, [&](int64_t row, int y, int64_t x, int cnt) {
        const int2 iv = __ldg(inside + y);
        float a[8], b[8];
        load8(g + row * nx + x, cnt, a);
        load8(e + row * nx + x, cnt, b);
        for (int i = 0; i < cnt; i++) {
            const unsigned int k = fkey(combined(a[i], b[i], gm, em));
            lo = min(lo, k);
            hi = max(hi, k);
            if (x + i >= iv.x && x + i < iv.y) {
                lo_in = min(lo_in, k);
                hi_in = max(hi_in, k);
            }
        }
    });
    lo = warp_min(lo);
    hi = warp_max(hi);
    lo_in = warp_min(lo_in);
    hi_in = warp_max(hi_in);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&st->cmin, lo);
        atomicMax(&st->cmax, hi);
        atomicMin(&st->cmin_in, lo_in);
        atomicMax(&st->cmax_in, hi_in);
    }
}

struct ConvertScalars {
    float gm, em, shift, denom, vmin, range;
};

__global__ void combined_convert(const uint16_t *__restrict__ g, const uint16_t *__restrict__ e,
                                 uint16_t *__restrict__ out, int64_t rows, int64_t ny, int64_t nx, bool vec,
                                 const int2 *__restrict__ inside, ConvertScalars s) {
    for_chunks(rows, ny, nx, vec, [&](int64_t row, int y, int64_t x, int cnt) {
        const int2 iv = __ldg(inside + y);
        float a[8], b[8];
        load8(g + row * nx + x, cnt, a);
        load8(e + row * nx + x, cnt, b);
        uint16_t q[8];
        for (int i = 0; i < cnt; i++) {
            const float c1 = __fdiv_rn(__fadd_rn(combined(a[i], b[i], s.gm, s.em), s.shift), s.denom);
            const float t = __fmul_rn(__fdiv_rn(__fsub_rn(c1, s.vmin), s.range), 65535.0f);
            const bool in = x + i >= iv.x && x + i < iv.y;
            q[i] = (in && s.range > 0.0f) ? (uint16_t) __float2uint_rz(t) : (uint16_t) 0;
        }
        if (cnt == 8) {
            uint4 w;
            w.x = q[0] | ((uint32_t) q[1] << 16);
            w.y = q[2] | ((uint32_t) q[3] << 16);
            w.z = q[4] | ((uint32_t) q[5] << 16);
            w.w = q[6] | ((uint32_t) q[7] << 16);
            *reinterpret_cast<uint4 *>(out + row * nx + x) = w;
        } else {
            out[row * nx + x] = q[0];
        }
    });
}

// numpy.linspace(-1, 1, n)[i] in FP64 (numpy: arange * step + start, last point = stop).
double linspace_pm1(int64_t i, int64_t n) {
    if (n == 1) return -1.0;
    if (i == n - 1) return 1.0;
    const double step = 2.0 / (double) (n - 1);
    volatile double t = (double) i * step;  // two roundings, as numpy (no fused multiply-add)
    return t + -1.0;
}

// Inside interval [x0, x1) of each row y of generate_cylinder_mask(ny, nx):
// xs[x]^2 + ys[y]^2 < 1 in FP64.  xs^2 falls then rises along x and fl(a + c) is
// monotone in a, so a row's inside voxels run from a first to a last index around
// the argmin of xs^2: two binary searches per row, exact.
void cylinder_intervals(int64_t ny, int64_t nx, std::vector<int2> &inside, bool &any_outside, bool &any_inside) {
    std::vector<double> xs2(nx);
    int64_t xm = 0;
    for (int64_t x = 0; x < nx; x++) {
        const double v = linspace_pm1(x, nx);
        volatile double sq = v * v;
        xs2[x] = sq;
        if (xs2[x] < xs2[xm]) xm = x;
    }
    inside.assign(ny, make_int2(0, 0));
    any_outside = any_inside = false;
    for (int64_t y = 0; y < ny; y++) {
        const double v = linspace_pm1(y, ny);
        volatile double ys2 = v * v;
        auto in = [&](int64_t x) {
            volatile double s = xs2[x] + ys2;
            return s < 1.0;
        };
        int64_t x0 = 0, x1 = 0;
        if (in(xm)) {
            int64_t lo = 0, hi = xm;  // first inside index in [0, xm]
            while (lo < hi) {
                const int64_t mid = (lo + hi) / 2;
                if (in(mid)) hi = mid;
                else lo = mid + 1;
            }
            x0 = lo;
            lo = xm + 1, hi = nx;  // first outside index in [xm + 1, nx]
            while (lo < hi) {
                const int64_t mid = (lo + hi) / 2;
                if (in(mid)) lo = mid + 1;
                else hi = mid;
            }
            x1 = lo;
        }
        inside[y] = make_int2((int) x0, (int) x1);
        any_outside |= x0 > 0 || x1 < nx;
        any_inside |= x1 > x0;
    }
}

// Zeroes the voxels of each row outside its cylinder interval (one block per row
// at a time; the inside voxels are neither read nor written).
__global__ void cylinder_zero(uint16_t *__restrict__ f, int64_t rows, int64_t ny, int nx,
                              const int2 *__restrict__ iv) {
    for (int64_t row = blockIdx.x; row < rows; row += gridDim.x) {
        const int2 in = __ldg(iv + row % ny);
        uint16_t *r = f + row * nx;
        for (int x = threadIdx.x; x < in.x; x += blockDim.x) r[x] = 0;
        for (int x = in.y + threadIdx.x; x < nx; x += blockDim.x) r[x] = 0;
    }
}

}  // namespace
}  // namespace maxi

using namespace maxi;

extern "C" int maxi_combine_fields(const uint16_t *gauss, const uint16_t *edt, int64_t nz, int64_t ny, int64_t nx,
                                   uint16_t *output, void *stream) {
    clear_error();
    if (!gauss || !edt || !output) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (nz <= 0 || ny <= 0 || nx <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "shape (%lld, %lld, %lld) has an empty axis", (long long) nz,
                         (long long) ny, (long long) nx);
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t rows = nz * ny;
    if (rows * nx >= (int64_t(1) << 32))
        return set_error(MAXI_ERR_UNSUPPORTED, "volumes of 2^32 voxels or more are not served by this step");

    std::vector<int2> inside;
    bool any_outside = false, any_inside = false;
    cylinder_intervals(ny, nx, inside, any_outside, any_inside);

    char *scratch = nullptr;
    const size_t iv_bytes = (size_t) ny * sizeof(int2);
    const size_t bytes = 256 + round_up((int64_t) iv_bytes, 256);
    if (cudaMallocAsync(reinterpret_cast<void **>(&scratch), bytes, st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of scratch", bytes);
    }
    CombineStats *d_st = reinterpret_cast<CombineStats *>(scratch);
    int2 *d_iv = reinterpret_cast<int2 *>(scratch + 256);
    CombineStats init{};
    init.cmin = init.cmin_in = 0xffffffffu;
    const bool vec = nx % 8 == 0 && ((reinterpret_cast<uintptr_t>(gauss) | reinterpret_cast<uintptr_t>(edt) |
                                       reinterpret_cast<uintptr_t>(output)) & 15) == 0;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t chunks = rows * (vec ? nx / 8 : nx);
    const unsigned grid = (unsigned) std::min<int64_t>(ceil_div(chunks, 256), (int64_t) sms * 16);
    const int threads = 256;
    CombineStats h{};
    auto finish = [&](int code) {
        cudaFreeAsync(scratch, st);
        return code;
    };
    cudaError_t e;
    if ((e = cudaMemcpyAsync(d_st, &init, sizeof(init), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_iv, inside.data(), iv_bytes, cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return finish(set_cuda_error(e, "combine_fields set-up"));
    field_maxima<<<grid, threads, 0, st>>>(gauss, edt, rows, ny, nx, vec, d_st);
    if ((e = cudaMemcpyAsync(&h, d_st, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return finish(set_cuda_error(e, "combine_fields maxima"));
    if (h.gmax == 0 || h.emax == 0)
        return finish(set_error(MAXI_ERR_INVALID_ARGUMENT,
                                "the %s field is all zero (the combination divides by its maximum)",
                                h.gmax == 0 ? "Gaussian" : "EDT"));
    const float gm = (float) h.gmax, em = (float) h.emax;
    combined_extremes<<<grid, threads, 0, st>>>(gauss, edt, rows, ny, nx, vec, d_iv, gm, em, d_st);
    if ((e = cudaMemcpyAsync(&h, d_st, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return finish(set_cuda_error(e, "combine_fields extremes"));

    // Scalar steps in FP32, in numpy's order (the x86-64 host rounds float
    // arithmetic to single precision).
    ConvertScalars s{};
    s.gm = gm;
    s.em = em;
    volatile float cmin = key_float(h.cmin), cmax = key_float(h.cmax);
    s.shift = std::fabs((float) cmin);
    volatile float denom = cmax + s.shift;
    s.denom = denom;
    float vmin = 0.0f, vmax = 0.0f;
    if (any_inside) {
        volatile float lo = key_float(h.cmin_in) + s.shift, hi = key_float(h.cmax_in) + s.shift;
        volatile float lo_d = lo / s.denom, hi_d = hi / s.denom;
        vmin = any_outside ? std::min(0.0f, (float) lo_d) : (float) lo_d;
        vmax = any_outside ? std::max(0.0f, (float) hi_d) : (float) hi_d;
    }
    s.vmin = vmin;
    volatile float range = vmax - vmin;
    s.range = range;
    combined_convert<<<grid, threads, 0, st>>>(gauss, edt, output, rows, ny, nx, vec, d_iv, s);
    e = cudaGetLastError();
    finish(0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "combine_fields convert");
}

extern "C" int maxi_mask_cylinder(uint16_t *field, int64_t nz, int64_t ny, int64_t nx, void *stream) {
    clear_error();
    if (!field) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (nz <= 0 || ny <= 0 || nx <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "shape (%lld, %lld, %lld) has an empty axis", (long long) nz,
                         (long long) ny, (long long) nx);
    if (nx >= (int64_t(1) << 31)) return set_error(MAXI_ERR_UNSUPPORTED, "rows of 2^31 voxels or more are not served");
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<int2> inside;
    bool any_outside = false, any_inside = false;
    cylinder_intervals(ny, nx, inside, any_outside, any_inside);
    if (!any_outside) return MAXI_OK;
    int2 *d_iv = nullptr;
    const size_t bytes = inside.size() * sizeof(int2);
    if (cudaMallocAsync(reinterpret_cast<void **>(&d_iv), bytes, st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of intervals", bytes);
    }
    cudaError_t e = cudaMemcpyAsync(d_iv, inside.data(), bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int64_t rows = nz * ny;
        const unsigned grid = (unsigned) std::min<int64_t>(rows, (int64_t) sms * 16);
        cylinder_zero<<<grid, 128, 0, st>>>(field, rows, ny, (int) nx, d_iv);
        e = cudaGetLastError();
    }
    cudaError_t e2 = cudaStreamSynchronize(st);  // the host intervals must outlive the copy
    cudaFreeAsync(d_iv, st);
    if (e == cudaSuccess) e = e2;
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "cylinder mask");
}
