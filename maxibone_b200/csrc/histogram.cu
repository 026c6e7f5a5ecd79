// 2-D (field value, voxel value) histogram of a voxel volume against a field:
// the reference's field_histogram (src/lib/cpp/cpu/histograms.cc:231-305, via
// src/pybind/histograms-pybind.cc:81-107), the consumer of the combined field
// in maxibone's pipeline (src/processing_steps/1000_compute_histograms.py:80-115).
//
// For every voxel (Z, Y, X) with Y >= y_start and X >= x_start: the voxel value v
// (uint16) counts as 0 outside [vmin, vmax] and is binned as
// floor((voxel_bins - 1) * ((v - vmin) / (vmax - vmin))) in FP64; the field is
// read at (min(nz - 1, floor(Z * nz/nZ)), floor(Y * ny/nY), floor(X * nx/nX))
// and binned the same way over [fmin, fmax]; pairs with a zero voxel or a zero
// field value are skipped; bins[field_bin][voxel_bin] += 1.
//
// Both values are uint16 and the coordinates depend on one axis each, so every
// FP64 expression is tabulated on the host (two 65536-entry bin maps, three axis
// maps) with the reference's own arithmetic; the kernel only gathers and counts.
// A warp adds equal bins once (match + popcount) before its 64-bit atomics.
// Field bins outside [0, field_bins) -- out-of-bounds writes in the reference --
// are skipped.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "host_util.h"

namespace maxi {
namespace {

// One block walks whole rows (Z, Y); its threads step along X.  Loop bounds are
// block-uniform, so every warp reaches the match below with all 32 lanes.
__global__ void field_histogram_kernel(const uint16_t *__restrict__ voxels, const uint16_t *__restrict__ field,
                                       int64_t nZ, int64_t nY, int nX, int64_t ny, int64_t nx, int64_t y_start,
                                       int x_start, const int32_t *__restrict__ vtab,
                                       const int32_t *__restrict__ ftab, const int32_t *__restrict__ zmap,
                                       const int32_t *__restrict__ ymap, const int32_t *__restrict__ xmap,
                                       unsigned long long *__restrict__ bins, int64_t voxel_bins) {
    const int lane = threadIdx.x & 31;
    for (int64_t row = blockIdx.x; row < nZ * nY; row += gridDim.x) {
        const int64_t Z = row / nY, Y = row - Z * nY;
        if (Y < y_start) continue;
        const uint16_t *vrow = voxels + row * nX;
        const uint16_t *frow = field + ((int64_t) __ldg(zmap + Z) * ny + __ldg(ymap + Y)) * nx;
        for (int X0 = x_start; X0 < nX; X0 += blockDim.x) {
            const int X = X0 + threadIdx.x;
            long long key = -1;
            if (X < nX) {
                const int32_t vb = __ldg(vtab + __ldg(vrow + X));
                if (vb >= 0) {
                    const int32_t fb = __ldg(ftab + __ldg(frow + __ldg(xmap + X)));
                    if (fb >= 0) key = (long long) fb * voxel_bins + vb;
                }
            }
            const unsigned same = __match_any_sync(0xffffffffu, key);
            if (key >= 0 && lane == __ffs(same) - 1) atomicAdd(bins + key, (unsigned long long) __popc(same));
        }
    }
}

// floor((bins - 1) * ((v - lo) / (hi - lo))) in FP64, as the reference writes it.
int64_t bin_of(double v, double lo, double hi, int64_t bins) {
    volatile double t = (v - lo) / (hi - lo);
    volatile double u = (double) (bins - 1) * t;
    return (int64_t) std::floor((double) u);
}

}  // namespace
}  // namespace maxi

using namespace maxi;

extern "C" int maxi_field_histogram(const uint16_t *voxels, int64_t nZ, int64_t nY, int64_t nX, const uint16_t *field,
                                    int64_t nz, int64_t ny, int64_t nx, int64_t y_start, int64_t x_start,
                                    uint64_t *bins, int64_t field_bins, int64_t voxel_bins, double vmin, double vmax,
                                    double fmin, double fmax, void *stream) {
    clear_error();
    if (!voxels || !field || !bins) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (nZ <= 0 || nY <= 0 || nX <= 0 || nz <= 0 || ny <= 0 || nx <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "empty voxel or field volume");
    if (field_bins <= 0 || voxel_bins <= 0 || field_bins * voxel_bins > (int64_t(1) << 34))
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "bad histogram size %lld x %lld", (long long) field_bins,
                         (long long) voxel_bins);
    if (!(vmax > vmin) || !(fmax > fmin))
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "empty value range");
    if (y_start < 0 || x_start < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "negative offset");
    if (nX >= (int64_t(1) << 31) || nx >= (int64_t(1) << 31))
        return set_error(MAXI_ERR_UNSUPPORTED, "rows of 2^31 voxels or more are not served");
    if (x_start >= nX || y_start >= nY) return MAXI_OK;  // nothing to count
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Tables with the reference's FP64 expressions (-1: the pair is not counted).
    std::vector<int32_t> tab(2 * 65536 + nZ + nY + nX);
    int32_t *vtab = tab.data(), *ftab = vtab + 65536, *zmap = ftab + 65536, *ymap = zmap + nZ, *xmap = ymap + nY;
    for (int v = 0; v < 65536; v++) {
        const double vv = (double) v;
        const double masked = (vv >= vmin && vv <= vmax) ? vv : 0.0;
        const int64_t b = bin_of(masked, vmin, vmax, voxel_bins);
        vtab[v] = (masked != 0.0 && b >= 0 && b < voxel_bins) ? (int32_t) b : -1;
        const int64_t fb = bin_of((double) v, fmin, fmax, field_bins);
        ftab[v] = (v > 0 && fb >= 0 && fb < field_bins) ? (int32_t) fb : -1;
    }
    const double dz = (double) nz / (double) nZ, dy = (double) ny / (double) nY, dx = (double) nx / (double) nX;
    for (int64_t Z = 0; Z < nZ; Z++) {
        volatile double t = (double) Z * dz;
        zmap[Z] = (int32_t) std::min<int64_t>(nz - 1, (int64_t) std::floor((double) t));
    }
    for (int64_t Y = 0; Y < nY; Y++) {
        volatile double t = (double) Y * dy;
        ymap[Y] = (int32_t) std::min<int64_t>(ny - 1, (int64_t) std::floor((double) t));
    }
    for (int64_t X = 0; X < nX; X++) {
        volatile double t = (double) X * dx;
        xmap[X] = (int32_t) std::min<int64_t>(nx - 1, (int64_t) std::floor((double) t));
    }

    int32_t *d_tab = nullptr;
    const size_t bytes = tab.size() * sizeof(int32_t);
    if (cudaMallocAsync(reinterpret_cast<void **>(&d_tab), bytes, st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of tables", bytes);
    }
    cudaError_t e = cudaMemcpyAsync(d_tab, tab.data(), bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const unsigned grid = (unsigned) std::min<int64_t>(nZ * nY, (int64_t) sms * 8);
        field_histogram_kernel<<<grid, 256, 0, st>>>(voxels, field, nZ, nY, (int) nX, ny, nx, y_start, (int) x_start, d_tab,
                                                     d_tab + 65536, d_tab + 2 * 65536, d_tab + 2 * 65536 + nZ,
                                                     d_tab + 2 * 65536 + nZ + nY,
                                                     reinterpret_cast<unsigned long long *>(bins), voxel_bins);
        e = cudaGetLastError();
    }
    // The host tables must outlive the copy.
    cudaError_t e2 = cudaStreamSynchronize(st);
    cudaFreeAsync(d_tab, st);
    if (e == cudaSuccess) e = e2;
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "field histogram");
}
