// The reference's histograms module on the GPU.
//
// field_histogram (src/lib/cpp/cpu/histograms.cc:231-305, via
// src/pybind/histograms-pybind.cc:81-107; the consumer of the diffusion field in
// src/processing_steps/1000_compute_histograms.py:470-472): for every voxel (Z, Y, X)
// with Y >= y_start and X >= x_start, the uint16 voxel value v counts as 0 outside
// [vmin, vmax] and is binned as floor((voxel_bins - 1) * ((v - vmin) / (vmax - vmin)))
// in FP64; the field is read at (min(nz - 1, floor(Z * nz/nZ)), floor(Y * ny/nY),
// floor(X * nx/nX)) and binned the same way over [fmin, fmax]; pairs with a zero
// voxel or a zero field value are skipped; bins[field_bin][voxel_bin] += 1.  Field
// bins outside [0, field_bins) -- out-of-bounds writes in the reference -- are skipped.
//
// axis_histograms (histograms.cc:14-80, via histograms-pybind.cc:30-66): each
// counted voxel of a z-block adds to x_bins[x], y_bins[y], z_bins[z] and
// r_bins[floor(sqrt((x-cx)^2 + (y-cy)^2))] at its voxel bin.
//
// Exact binning without FP64 in the kernels.  Each bin expression is a monotone
// function of an integer value, so the host evaluates it with the reference's own
// FP64 arithmetic for all 65536 values and keeps, per bin b, the threshold T[b] =
// the smallest counted value whose bin is >= b.  A kernel estimates the bin in FP32
// from the value's offset in the counted range and settles it with one comparison
// each way against T (T[b] <= v < T[b+1] holds for exactly one b).  The host checks,
// before any launch, that the estimate is within one bin for every counted value, so
// the result is the reference's bin.  The tables are (bins + 1) words, L1-resident.
//
// Counting.  One thread takes 8 consecutive voxels of a row (one 16-byte load when
// rows are 16-byte aligned) and adds runs of equal keys once.  field_histogram
// issues one 64-bit reduction per run into the histogram (L2-resident at the
// pipeline's 2048 x 4096); each of its blocks walks one contiguous range of rows.  axis_histograms counts each row's voxel bins in a
// shared-memory histogram with a list of the bins it touched, then adds those to
// y_bins[y] and z_bins[z]; x and radial bins take one reduction per voxel.
#include <cmath>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "host_util.h"

namespace maxi {
namespace {

constexpr int kVec = 8;  // voxels per thread (one 16-byte load)

// A counted value range [lo, lo + span] and its bin thresholds.
struct BinMap {
    const uint32_t *T;  // T[0 .. bins]
    int lo, span, bins;
    float a, c;  // estimate: (v - lo) * a + c
};

// The bin of v, or -1 if v is not counted.
__device__ __forceinline__ int bin_of(const BinMap &m, int v) {
    const unsigned d = (unsigned) (v - m.lo);
    if (d > (unsigned) m.span) return -1;
    int b = __float2int_rz(__fmaf_rn((float) d, m.a, m.c));
    b = min(max(b, 0), m.bins - 1);
    if ((uint32_t) v < __ldg(m.T + b)) b--;
    else if ((uint32_t) v >= __ldg(m.T + b + 1)) b++;
    return b;
}

// Voxels are read once: loaded evict-first, so the L2-resident bins stay in L2.
__device__ __forceinline__ void load_row8(const uint16_t *p, int (&v)[kVec]) {
    const uint4 w = __ldcs(reinterpret_cast<const uint4 *>(p));
    const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        v[2 * k] = (int) (u[k] & 0xffffu);
        v[2 * k + 1] = (int) (u[k] >> 16);
    }
}

// VEC8: rows are 16-byte aligned (nX % 8 == 0, aligned base); otherwise one voxel at a time.
template <bool VEC8>
__global__ void field_histogram_kernel(const uint16_t *__restrict__ voxels, const uint16_t *__restrict__ field,
                                       int64_t nZ, int64_t nY, int nX, int64_t ny, int64_t nx, int64_t y_start,
                                       int x_start, BinMap vm, BinMap fm, const int32_t *__restrict__ zmap,
                                       const int32_t *__restrict__ ymap, const int32_t *__restrict__ xmap,
                                       unsigned long long *__restrict__ bins, int64_t voxel_bins) {
    constexpr int V = VEC8 ? kVec : 1;
    const int x_first = x_start / V * V;
    // Each block takes one contiguous range of rows, so the blocks at work at any time
    // sit far apart in the volume: a smooth field gives neighbouring rows the same
    // keys, and same-address reductions from many blocks at once serialise in L2.
    const int64_t rows = nZ * nY, per = (rows + gridDim.x - 1) / gridDim.x;
    const int64_t row_end = min(rows, (int64_t) (blockIdx.x + 1) * per);
    for (int64_t row = (int64_t) blockIdx.x * per; row < row_end; row++) {
        const int64_t Z = row / nY, Y = row - Z * nY;
        if (Y < y_start) continue;
        const uint16_t *vrow = voxels + row * nX;
        const uint16_t *frow = field + ((int64_t) __ldg(zmap + Z) * ny + __ldg(ymap + Y)) * nx;
        for (int X = x_first + threadIdx.x * V; X < nX; X += blockDim.x * V) {
            int v[V];
            if constexpr (VEC8) load_row8(vrow + X, v);
            else v[0] = __ldcs(vrow + X);
            long long run_key = -1;
            unsigned run = 0;
#pragma unroll
            for (int j = 0; j < V; j++) {
                const int x = X + j;
                long long key = -1;
                const int vb = x >= x_start ? bin_of(vm, v[j]) : -1;
                if (vb >= 0) {
                    const int fb = bin_of(fm, __ldg(frow + __ldg(xmap + x)));
                    if (fb >= 0) key = (long long) fb * voxel_bins + vb;
                }
                if (key == run_key) {
                    run++;
                } else {
                    if (run_key >= 0) atomicAdd(bins + run_key, (unsigned long long) run);
                    run_key = key;
                    run = 1;
                }
            }
            if (run_key >= 0) atomicAdd(bins + run_key, (unsigned long long) run);
        }
    }
}

// floor(sqrt(n)) for 0 <= n < 2^50: a float estimate corrected in integers.  In that
// range it equals floor of the correctly rounded double sqrt of n, the reference's
// std::floor(std::sqrt(uint64)), since (k + 1)^2 - 1 and (k + 1)^2 stay apart in double.
__device__ __forceinline__ int64_t isqrt64(int64_t n) {
    int64_t r = (int64_t) sqrtf((float) n);
    while (r * r > n) r--;
    while ((r + 1) * (r + 1) <= n) r++;
    return r;
}

// PRIV: the block keeps a shared histogram of the current row's voxel bins
// (voxel_bins counters + voxel_bins touched-bin slots + a count) and adds it to
// y_bins[y] and z_bins[z] at the end of the row; otherwise every voxel adds directly.
// The row loop is block-uniform (it holds barriers).
template <bool VEC8, bool PRIV>
__global__ void axis_histograms_kernel(const uint16_t *__restrict__ voxels, int64_t nzl, int64_t Ny, int Nx,
                                       int64_t z_start, int64_t y_start, int x_start, BinMap vm, int64_t cy,
                                       int64_t cx, unsigned long long *__restrict__ x_bins,
                                       unsigned long long *__restrict__ y_bins,
                                       unsigned long long *__restrict__ z_bins,
                                       unsigned long long *__restrict__ r_bins, int voxel_bins, int64_t n_r) {
    constexpr int V = VEC8 ? kVec : 1;
    extern __shared__ uint32_t sh[];
    uint32_t *hist = sh, *touched = sh + voxel_bins, *n_touched = sh + 2 * voxel_bins;
    if (PRIV) {
        for (int i = threadIdx.x; i < voxel_bins; i += blockDim.x) hist[i] = 0;
        if (threadIdx.x == 0) *n_touched = 0;
        __syncthreads();
    }
    const int x_first = x_start / V * V;
    for (int64_t row = blockIdx.x; row < nzl * Ny; row += gridDim.x) {
        const int64_t zl = row / Ny, y = row - zl * Ny;
        if (y < y_start) continue;
        const uint16_t *vrow = voxels + row * Nx;
        const int64_t dy2 = (y - cy) * (y - cy);
        unsigned long long *yrow = y_bins + y * voxel_bins, *zrow = z_bins + (z_start + zl) * voxel_bins;
        for (int X = x_first + threadIdx.x * V; X < Nx; X += blockDim.x * V) {
            int v[V];
            if constexpr (VEC8) load_row8(vrow + X, v);
            else v[0] = __ldcs(vrow + X);
            long long r_key = -1;
            unsigned r_run = 0;
            int b_key = -1;
            unsigned b_run = 0;
#pragma unroll
            for (int j = 0; j < V; j++) {
                const int x = X + j;
                const int vb = x >= x_start ? bin_of(vm, v[j]) : -1;
                long long rk = -1;
                if (vb >= 0) {
                    atomicAdd(x_bins + (int64_t) x * voxel_bins + vb, 1ull);
                    const int64_t r = isqrt64(dy2 + (x - cx) * (x - cx));
                    if (r < n_r) rk = r * voxel_bins + vb;
                    if (PRIV) {
                        if (atomicAdd(hist + vb, 1u) == 0) touched[atomicAdd(n_touched, 1u)] = (uint32_t) vb;
                    }
                }
                if (rk == r_key) {
                    r_run++;
                } else {
                    if (r_key >= 0) atomicAdd(r_bins + r_key, (unsigned long long) r_run);
                    r_key = rk;
                    r_run = 1;
                }
                if (!PRIV) {
                    if (vb == b_key) {
                        b_run++;
                    } else {
                        if (b_key >= 0) {
                            atomicAdd(yrow + b_key, (unsigned long long) b_run);
                            atomicAdd(zrow + b_key, (unsigned long long) b_run);
                        }
                        b_key = vb;
                        b_run = 1;
                    }
                }
            }
            if (r_key >= 0) atomicAdd(r_bins + r_key, (unsigned long long) r_run);
            if (!PRIV && b_key >= 0) {
                atomicAdd(yrow + b_key, (unsigned long long) b_run);
                atomicAdd(zrow + b_key, (unsigned long long) b_run);
            }
        }
        if (PRIV) {
            __syncthreads();
            const uint32_t n = *n_touched;
            for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
                const uint32_t b = touched[i];
                const unsigned long long c = hist[b];
                hist[b] = 0;
                atomicAdd(yrow + b, c);
                atomicAdd(zrow + b, c);
            }
            __syncthreads();
            if (threadIdx.x == 0) *n_touched = 0;
            __syncthreads();
        }
    }
}

// floor((bins - 1) * ((v - lo) / (hi - lo))) in FP64, as the reference writes it.
int64_t ref_bin(double v, double lo, double hi, int64_t bins) {
    volatile double t = (v - lo) / (hi - lo);
    volatile double u = (double) (bins - 1) * t;
    return (int64_t) std::floor((double) u);
}

// Thresholds of an exact bin table (-1: not counted) whose counted values form one
// contiguous range with bins non-decreasing in the value; checks the FP32 estimate.
// `scale` and `origin` are the FP64 slope and zero of the bin expression.
int make_bin_map(const std::vector<int32_t> &tab, int64_t bins, double scale, double origin,
                 std::vector<uint32_t> &T, BinMap &m, const char *what) {
    int lo = -1, hi = -1;
    for (int v = 0; v < 65536; v++)
        if (tab[v] >= 0) {
            if (lo < 0) lo = v;
            hi = v;
        }
    T.assign(bins + 1, 0);
    m.bins = (int) bins;
    if (lo < 0) {  // nothing counted: a range no uint16 reaches
        m.lo = 65536 + 1;
        m.span = 0;
        m.a = m.c = 0.0f;
        return MAXI_OK;
    }
    for (int v = lo; v <= hi; v++)
        if (tab[v] < 0 || (v > lo && tab[v] < tab[v - 1]))
            return set_error(MAXI_ERR_UNSUPPORTED, "%s bins are not monotone in the value", what);
    m.lo = lo;
    m.span = hi - lo;
    m.a = (float) scale;
    m.c = (float) (((double) lo - origin) * scale);
    int64_t b = 0;
    for (int v = lo; v <= hi; v++)
        while (b <= tab[v]) T[b++] = (uint32_t) v;
    while (b <= bins) T[b++] = (uint32_t) hi + 1;
    for (int v = lo; v <= hi; v++) {
        int est = (int) std::fmaf((float) (v - lo), m.a, m.c);
        est = std::min(std::max(est, 0), m.bins - 1);
        if (std::abs(est - tab[v]) > 1)
            return set_error(MAXI_ERR_UNSUPPORTED, "%s bin estimate off by more than one at value %d", what, v);
    }
    return MAXI_OK;
}

// Bin of every uint16 value, -1 where the reference does not count it.  Voxels:
// values outside [lo, hi] count as 0 and zero voxels are skipped.  Field values:
// zero values and bins outside [0, bins) are skipped.
void value_table(std::vector<int32_t> &tab, bool voxel, double lo, double hi, int64_t bins) {
    tab.assign(65536, -1);
    for (int v = 1; v < 65536; v++) {
        const double vv = (double) v;
        if (voxel && !(vv >= lo && vv <= hi)) continue;
        const int64_t b = ref_bin(vv, lo, hi, bins);
        if (b >= 0 && b < bins) tab[v] = (int32_t) b;
    }
}

// The bin map of (kind, lo, hi, bins), built once and kept: the pipeline calls the
// histograms block by block with the same ranges.  A few recent maps are kept.
struct CachedMap {
    bool voxel;
    double lo, hi;
    int64_t bins;
    std::vector<uint32_t> T;
    BinMap m;
};

int cached_bin_map(bool voxel, double lo, double hi, int64_t bins, std::vector<uint32_t> &T, BinMap &m) {
    static std::mutex mu;
    static std::vector<CachedMap> cache;
    std::lock_guard<std::mutex> lock(mu);
    for (const CachedMap &c : cache)
        if (c.voxel == voxel && c.lo == lo && c.hi == hi && c.bins == bins) {
            T = c.T;
            m = c.m;
            return MAXI_OK;
        }
    std::vector<int32_t> tab;
    value_table(tab, voxel, lo, hi, bins);
    const int rc = make_bin_map(tab, bins, (double) (bins - 1) / (hi - lo), lo, T, m, voxel ? "voxel" : "field");
    if (rc) return rc;
    if (cache.size() >= 4) cache.erase(cache.begin());
    cache.push_back({voxel, lo, hi, bins, T, m});
    return MAXI_OK;
}

int sm_count() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Device copy of host words laid out in 16-byte aligned segments.
struct DeviceTables {
    std::vector<uint32_t> host;
    uint32_t *dev = nullptr;
    size_t add(const uint32_t *p, size_t n) {
        const size_t at = host.size();
        host.insert(host.end(), p, p + n);
        host.resize((host.size() + 3) / 4 * 4, 0);
        return at;
    }
};

int upload(DeviceTables &t, cudaStream_t st) {
    const size_t bytes = t.host.size() * sizeof(uint32_t);
    if (cudaMallocAsync(reinterpret_cast<void **>(&t.dev), bytes, st) != cudaSuccess) {
        cudaGetLastError();
        t.dev = nullptr;
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of tables", bytes);
    }
    cudaError_t e = cudaMemcpyAsync(t.dev, t.host.data(), bytes, cudaMemcpyHostToDevice, st);
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "histogram tables");
}

// Waits for the launch (the host tables must outlive their copy) and frees the device copy.
int finish(DeviceTables &t, cudaStream_t st, int rc, const char *what) {
    cudaError_t e = rc == MAXI_OK ? cudaGetLastError() : cudaSuccess;
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (t.dev) cudaFreeAsync(t.dev, st);
    if (rc != MAXI_OK) return rc;
    if (e == cudaSuccess) e = e2;
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, what);
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
    if (field_bins <= 0 || voxel_bins <= 0 || field_bins > (1 << 20) || voxel_bins > (1 << 20))
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "bad histogram size %lld x %lld", (long long) field_bins,
                         (long long) voxel_bins);
    if (!(vmax > vmin) || !(fmax > fmin)) return set_error(MAXI_ERR_INVALID_ARGUMENT, "empty value range");
    if (y_start < 0 || x_start < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "negative offset");
    if (nX >= (int64_t(1) << 30) || nx >= (int64_t(1) << 31))
        return set_error(MAXI_ERR_UNSUPPORTED, "rows of 2^30 voxels or more are not served");
    if (x_start >= nX || y_start >= nY) return MAXI_OK;  // nothing to count
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    std::vector<uint32_t> vT, fT;
    BinMap vm{}, fm{};
    if ((rc = cached_bin_map(true, vmin, vmax, voxel_bins, vT, vm))) return rc;
    if ((rc = cached_bin_map(false, fmin, fmax, field_bins, fT, fm))) return rc;
    std::vector<uint32_t> zmap(nZ), ymap(nY), xmap(nX);
    const double dz = (double) nz / (double) nZ, dy = (double) ny / (double) nY, dx = (double) nx / (double) nX;
    for (int64_t Z = 0; Z < nZ; Z++) {
        volatile double t = (double) Z * dz;
        zmap[Z] = (uint32_t) std::min<int64_t>(nz - 1, (int64_t) std::floor((double) t));
    }
    for (int64_t Y = 0; Y < nY; Y++) {
        volatile double t = (double) Y * dy;
        ymap[Y] = (uint32_t) std::min<int64_t>(ny - 1, (int64_t) std::floor((double) t));
    }
    for (int64_t X = 0; X < nX; X++) {
        volatile double t = (double) X * dx;
        xmap[X] = (uint32_t) std::min<int64_t>(nx - 1, (int64_t) std::floor((double) t));
    }
    DeviceTables t;
    const size_t o_vT = t.add(vT.data(), vT.size()), o_fT = t.add(fT.data(), fT.size());
    const size_t o_z = t.add(zmap.data(), zmap.size()), o_y = t.add(ymap.data(), ymap.size());
    const size_t o_x = t.add(xmap.data(), xmap.size());
    rc = upload(t, st);
    if (rc == MAXI_OK) {
        vm.T = t.dev + o_vT;
        fm.T = t.dev + o_fT;
        const int32_t *zm = reinterpret_cast<const int32_t *>(t.dev + o_z);
        const int32_t *ym = reinterpret_cast<const int32_t *>(t.dev + o_y);
        const int32_t *xm = reinterpret_cast<const int32_t *>(t.dev + o_x);
        auto *b = reinterpret_cast<unsigned long long *>(bins);
        const bool vec = nX % kVec == 0 && reinterpret_cast<uintptr_t>(voxels) % 16 == 0;
        const unsigned grid = (unsigned) std::min<int64_t>(nZ * nY, (int64_t) sm_count() * 16);
        if (vec)
            field_histogram_kernel<true><<<grid, 128, 0, st>>>(voxels, field, nZ, nY, (int) nX, ny, nx, y_start,
                                                               (int) x_start, vm, fm, zm, ym, xm, b, voxel_bins);
        else
            field_histogram_kernel<false><<<grid, 256, 0, st>>>(voxels, field, nZ, nY, (int) nX, ny, nx, y_start,
                                                                (int) x_start, vm, fm, zm, ym, xm, b, voxel_bins);
    }
    return finish(t, st, rc, "field histogram");
}

extern "C" int maxi_axis_histograms(const uint16_t *voxels, int64_t nz_block, int64_t Nz, int64_t Ny, int64_t Nx,
                                    int64_t z_start, int64_t y_start, int64_t x_start, uint64_t *x_bins,
                                    uint64_t *y_bins, uint64_t *z_bins, uint64_t *r_bins, int64_t voxel_bins,
                                    int64_t n_r, int64_t cy, int64_t cx, double vmin, double vmax, void *stream) {
    clear_error();
    if (!voxels || !x_bins || !y_bins || !z_bins || !r_bins) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (nz_block <= 0 || Nz <= 0 || Ny <= 0 || Nx <= 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "empty volume");
    if (voxel_bins <= 0 || voxel_bins > (1 << 20) || n_r <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "bad histogram size");
    if (!(vmax > vmin)) return set_error(MAXI_ERR_INVALID_ARGUMENT, "empty value range");
    if (z_start < 0 || y_start < 0 || x_start < 0 || cy < 0 || cx < 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "negative offset or centre");
    if (Nx >= (int64_t(1) << 30)) return set_error(MAXI_ERR_UNSUPPORTED, "rows of 2^30 voxels or more are not served");
    // Largest distance from the centre; the integer square root equals the reference's double one below 2^50.
    const int64_t ry = std::max(cy, Ny - 1 - cy), rx = std::max(cx, Nx - 1 - cx);
    if (ry >= (int64_t(1) << 24) || rx >= (int64_t(1) << 24))
        return set_error(MAXI_ERR_UNSUPPORTED, "distances of 2^24 voxels or more from the centre are not served");
    const int64_t nzl = std::min(z_start + nz_block, Nz) - z_start;
    if (nzl <= 0 || y_start >= Ny || x_start >= Nx) return MAXI_OK;  // nothing to count
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    std::vector<uint32_t> vT;
    BinMap vm{};
    if ((rc = cached_bin_map(true, vmin, vmax, voxel_bins, vT, vm))) return rc;
    DeviceTables t;
    const size_t o_vT = t.add(vT.data(), vT.size());
    rc = upload(t, st);
    if (rc == MAXI_OK) {
        vm.T = t.dev + o_vT;
        auto *xb = reinterpret_cast<unsigned long long *>(x_bins), *yb = reinterpret_cast<unsigned long long *>(y_bins);
        auto *zb = reinterpret_cast<unsigned long long *>(z_bins), *rb = reinterpret_cast<unsigned long long *>(r_bins);
        const bool vec = Nx % kVec == 0 && reinterpret_cast<uintptr_t>(voxels) % 16 == 0;
        const int threads = vec ? 128 : 256;
        // Row privatisation: 2 * voxel_bins + 1 words of shared memory, up to 8192 bins.
        const bool priv = voxel_bins <= 8192;
        const size_t smem = priv ? (2 * (size_t) voxel_bins + 1) * sizeof(uint32_t) : 0;
        const unsigned grid = (unsigned) std::min<int64_t>(nzl * Ny, (int64_t) sm_count() * 16);
        auto launch = [&](auto kern) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
            if (e != cudaSuccess) return set_cuda_error(e, "axis histograms set-up");
            kern<<<grid, threads, smem, st>>>(voxels, nzl, Ny, (int) Nx, z_start, y_start, (int) x_start, vm, cy, cx,
                                              xb, yb, zb, rb, (int) voxel_bins, n_r);
            return (int) MAXI_OK;
        };
        if (vec) rc = priv ? launch(axis_histograms_kernel<true, true>) : launch(axis_histograms_kernel<true, false>);
        else rc = priv ? launch(axis_histograms_kernel<false, true>) : launch(axis_histograms_kernel<false, false>);
    }
    return finish(t, st, rc, "axis histograms");
}
