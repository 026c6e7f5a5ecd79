// Single-volume tensor-core passes for 16-bit field storage (BF16 / FP16):
// host side of the kernels in tc_kernels.cuh (tensor maps with the volume's
// shape, one persistent launch per pass, one CTA per SM).
#include <cudaTypedefs.h>

#include <mutex>

#include "host_util.h"
#include "profiler.h"
#include "tc_kernels.cuh"
#include "tc_yx.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

namespace maxi {
namespace tc {

// ---- host side -----------------------------------------------------------------

PFN_cuTensorMapEncodeTiled_v12000 tc_encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

static uint16_t bits_bf16(float v) { return __bfloat16_as_ushort(__float2bfloat16_rn(v)); }
static float from_bf16(uint16_t b) { return __bfloat162float(__ushort_as_bfloat16(b)); }
static uint16_t bits_f16(float v) { return __half_as_ushort(__float2half_rn(v)); }
static float from_f16(uint16_t b) { return __half2float(__ushort_as_half(b)); }


bool tc_supported(int radius, int64_t nz, int64_t ny, int64_t nx) {
    if (radius < 1 || radius > kTcMaxRadiusWide) return false;
    if (nx % 8 != 0 || nx < 64) return false;  // TMA: 16-byte row strides, at least one 64-wide box
    if (nz > INT32_MAX / 2 || ny > INT32_MAX / 2 || nx > INT32_MAX / 2) return false;
    if (nz * ny >= (int64_t(1) << 31)) return false;  // rows and tile indices fit 32-bit arithmetic
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return major == 10 && tc_encode_fn() != nullptr;
}

template <typename S>
cudaError_t tc_strided(const S *in, S *out, int64_t nz, int64_t ny, int64_t nx, bool axis_z, const float *kernel,
                       int radius, bool error_feedback, cudaStream_t st, const YzRows *in_rows, bool hi_only) {
    if (!axis_z) in_rows = nullptr;
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    const int tn = strided_tn(radius), stages = kStridedStages;
    StridedLaunch<OneVolumeStrided> p{};
    fill_pass_taps(p.taps, kernel, radius, 0, (int) round_up(kTM + 2 * radius, 16), is_bf16, error_feedback, hi_only);
    OneVolumeStrided &sc = p.sched;
    sc.out = out;
    sc.nx = nx;
    sc.tn = tn;
    int64_t n_other;
    if (axis_z) { sc.A = nz; n_other = ny; sc.stride_a = ny * nx; sc.stride_o = nx; }
    else { sc.A = ny; n_other = nz; sc.stride_a = nx; sc.stride_o = ny * nx; }
    sc.n_at = (int) ceil_div(sc.A, kTM);
    sc.n_xc = (int) ceil_div(nx, tn);
    sc.n_cols = (int64_t) sc.n_xc * n_other;
    sc.in_rows = (!axis_z || in_rows) ? 1 : 0;

    CUtensorMap map;
    const CUtensorMapDataType dt = is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) ny, (cuuint64_t) nz};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * ny * 2)};
    const cuuint32_t brows = (cuuint32_t) p.taps.box_rows;
    const cuuint32_t box[3] = {64u, axis_z ? 1u : brows, axis_z ? brows : 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    // z pass over [y][z][x] rows: dims (x, z, y), rows nx apart, y slabs nz_total * nx apart.
    const cuuint64_t rdims[3] = {(cuuint64_t) nx, (cuuint64_t) nz, (cuuint64_t) ny};
    const cuuint64_t rstrides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (in_rows ? in_rows->nz_total * nx * 2 : 0)};
    const cuuint32_t rbox[3] = {64u, brows, 1u};
    void *in_base = in_rows ? static_cast<void *>(static_cast<S *>(in_rows->base) + in_rows->z0 * nx)
                            : static_cast<void *>(const_cast<S *>(in));
    CUresult cr = tc_encode_fn()(&map, dt, 3, in_base, in_rows ? rdims : dims, in_rows ? rstrides : strides,
                                 in_rows ? rbox : box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    CUtensorMap map_out = map;  // the z pass stores without a map
    if (!axis_z) {
        const cuuint32_t obox[3] = {32u, 32u, 1u};
        cr = tc_encode_fn()(&map_out, dt, 3, out, dims, strides, obox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                            CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    if (2 * tn + 2 * p.taps.kcols > (int) kTmemColsStrided) return cudaErrorInvalidValue;
    const int smem = strided_smem_bytes(p.taps.kp, tn, stages);
    auto *kern = tn == 128 ? (axis_z ? tc_strided_kernel<S, true, 128, OneVolumeStrided>
                                     : tc_strided_kernel<S, false, 128, OneVolumeStrided>)
                           : (axis_z ? tc_strided_kernel<S, true, 64, OneVolumeStrided>
                                     : tc_strided_kernel<S, false, 64, OneVolumeStrided>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(sc.n_cols, sms);
    kern<<<(unsigned) grid, kThreads, smem, st>>>(map, map_out, p);
    return cudaGetLastError();
}

template cudaError_t tc_strided<__nv_bfloat16>(const __nv_bfloat16 *, __nv_bfloat16 *, int64_t, int64_t, int64_t,
                                               bool, const float *, int, bool, cudaStream_t, const YzRows *, bool);
template cudaError_t tc_strided<__half>(const __half *, __half *, int64_t, int64_t, int64_t, bool, const float *, int,
                                        bool, cudaStream_t, const YzRows *, bool);

void tc_split_taps(const float *kernel, int radius, bool is_bf16, float scale, uint16_t *hi, uint16_t *lo) {
    for (int i = 0; i < 2 * radius + 1; i++) {
        const float k = kernel[i] * scale;
        if (is_bf16) {
            hi[i] = bits_bf16(k);
            lo[i] = bits_bf16(k - from_bf16(hi[i]));
        } else {
            hi[i] = bits_f16(k);
            lo[i] = bits_f16(k - from_f16(hi[i]));
        }
    }
}

// Neighbour of a finite 16-bit float (bit pattern b) towards +inf (up) or -inf.
static uint16_t step16(uint16_t b, bool up) {
    const bool neg = (b & 0x8000u) != 0;
    if ((b & 0x7fffu) == 0) return up ? 0x0001u : 0x8001u;  // +-0 -> smallest subnormal of that direction
    return (uint16_t) ((up != neg) ? b + 1 : b - 1);
}

void tc_round_taps_matched(const float *kernel, int radius, bool is_bf16, float scale, uint16_t *out) {
    const int n = 2 * radius + 1;
    auto from = [&](uint16_t b) { return (double) (is_bf16 ? from_bf16(b) : from_f16(b)); };
    std::vector<double> k(n), d0(n), d1(n);
    std::vector<uint16_t> b0(n), b1(n);
    for (int i = 0; i < n; i++) {
        const float v = kernel[i] * scale;
        k[i] = (double) v;
        b0[i] = is_bf16 ? bits_bf16(v) : bits_f16(v);
        const double q = from(b0[i]);
        b1[i] = q == k[i] ? b0[i] : step16(b0[i], q < k[i]);
        d0[i] = q - k[i];
        d1[i] = from(b1[i]) - k[i];
    }
    // Groups flipped together: the symmetric pairs (r - j, r + j) of a
    // symmetric kernel keep it symmetric; otherwise every tap alone.
    bool sym = true;
    for (int j = 1; j <= radius; j++) sym = sym && kernel[radius - j] == kernel[radius + j];
    std::vector<std::vector<int>> groups;
    if (sym) {
        groups.push_back({radius});
        for (int j = 1; j <= radius; j++) groups.push_back({radius - j, radius + j});
    } else {
        for (int i = 0; i < n; i++) groups.push_back({i});
    }
    const int G = (int) groups.size();
    std::vector<double> g0(G), g2(G);  // change of the sum / second moment when group g flips
    double s0 = 0.0, s2 = 0.0;         // current errors of the sum and second moment
    for (int i = 0; i < n; i++) {
        const double j2 = (double) (i - radius) * (i - radius);
        s0 += d0[i];
        s2 += j2 * d0[i];
    }
    for (int g = 0; g < G; g++)
        for (int i : groups[g]) {
            const double j2 = (double) (i - radius) * (i - radius);
            g0[g] += d1[i] - d0[i];
            g2[g] += j2 * (d1[i] - d0[i]);
        }
    const double w2 = 1.0 / std::max(1.0, (double) radius * radius);
    auto cost = [&](double a, double b) { return std::fabs(a) + w2 * std::fabs(b); };
    std::vector<int> flip(G, 0);
    // Greedy local search over single and paired group flips; each accepted
    // move lowers the cost, so it ends.
    for (int iter = 0; iter < 4 * G; iter++) {
        double best = cost(s0, s2);
        int bi = -1, bj = -1;
        for (int a = 0; a < G; a++) {
            if (g0[a] == 0.0 && g2[a] == 0.0) continue;
            const double sa = flip[a] ? -1.0 : 1.0;
            const double c1 = cost(s0 + sa * g0[a], s2 + sa * g2[a]);
            if (c1 < best) { best = c1; bi = a; bj = -1; }
            for (int b = a + 1; b < G; b++) {
                const double sb = flip[b] ? -1.0 : 1.0;
                const double c2 = cost(s0 + sa * g0[a] + sb * g0[b], s2 + sa * g2[a] + sb * g2[b]);
                if (c2 < best) { best = c2; bi = a; bj = b; }
            }
        }
        if (bi < 0) break;
        for (int g : {bi, bj}) {
            if (g < 0) continue;
            const double sg = flip[g] ? -1.0 : 1.0;
            s0 += sg * g0[g];
            s2 += sg * g2[g];
            flip[g] ^= 1;
        }
    }
    for (int g = 0; g < G; g++)
        for (int i : groups[g]) out[i] = flip[g] ? b1[i] : b0[i];
}

float tc_round_taps_scaled(const float *kernel, int radius, bool is_bf16, float base_scale, uint16_t *out) {
    const int n = 2 * radius + 1;
    // Results per kernel (the search costs milliseconds; launches repeat it).
    static std::mutex mu;
    static std::map<std::vector<uint32_t>, std::pair<float, std::vector<uint16_t>>> cache;
    std::vector<uint32_t> key(n + 2);
    key[0] = (uint32_t) is_bf16;
    std::memcpy(&key[1], &base_scale, 4);
    std::memcpy(&key[2], kernel, 4 * (size_t) n);
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = cache.find(key);
        if (it != cache.end()) {
            std::copy(it->second.second.begin(), it->second.second.end(), out);
            return it->second.first;
        }
    }
    auto from = [&](uint16_t b) { return (double) (is_bf16 ? from_bf16(b) : from_f16(b)); };
    double sum = 0.0, m2 = 0.0;
    for (int i = 0; i < n; i++) {
        sum += kernel[i];
        m2 += (double) (i - radius) * (i - radius) * kernel[i];
    }
    const double w2 = 0.01 / std::max(1.0, (double) radius * radius);
    // Candidate scales base x (1 + c / C): fewer for wide kernels, whose search is slower.
    const int C = radius <= 32 ? 256 : radius <= 64 ? 32 : 1;
    std::vector<uint16_t> bits(n), best_bits(n);
    float best_s = base_scale;
    double best_cost = -1.0;
    for (int c = 0; c < C; c++) {
        const float sc = base_scale * (1.0f + (float) c / (float) C);
        tc_round_taps_matched(kernel, radius, is_bf16, sc, bits.data());
        const double inv = (double) (1.0f / sc);  // the factor the epilogues apply
        double s0 = 0.0, s2 = 0.0;
        for (int i = 0; i < n; i++) {
            const double q = from(bits[i]) * inv;
            s0 += q;
            s2 += (double) (i - radius) * (i - radius) * q;
        }
        const double cost = std::fabs(s0 - sum) + w2 * std::fabs(s2 - m2);
        if (best_cost < 0.0 || cost < best_cost) {
            best_cost = cost;
            best_s = sc;
            best_bits = bits;
        }
    }
    std::copy(best_bits.begin(), best_bits.end(), out);
    std::lock_guard<std::mutex> lk(mu);
    cache[key] = {best_s, best_bits};
    return best_s;
}

bool tc_yx_supported(int radius, int64_t nz, int64_t ny, int64_t nx) {
    return radius <= kTcMaxRadius && tc_supported(radius, nz, ny, nx) &&
           nz * ceil_div(ny, kTM) * ceil_div(nx, kXTN) < (int64_t(1) << 31);
}

template <typename S>
cudaError_t tc_yx(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass, uint16_t *out_u16,
                  float *field_out, int64_t nz, int64_t ny, int64_t nx, const float *kernel, int radius,
                  bool error_feedback, bool hi_only, cudaStream_t st, const YzRows *out_rows) {
    if (radius > kTcMaxRadius) return cudaErrorInvalidValue;
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    if (final_pass) out_rows = nullptr;
    YxLaunch<OneVolumeYx> p{};
    const int ra = (int) round_up(radius, 8);
    if (!hi_only) return cudaErrorInvalidValue;  // the fused kernel holds one coefficient set
    fill_pass_taps(p.t, kernel, radius, ra, (int) round_up(kXTN + ra + radius, 16), is_bf16, error_feedback, true);
    if (p.t.kp > kYxMaxCols || (uint32_t) p.t.kp / 2 > kYxYpCols) return cudaErrorInvalidValue;
    p.final_pass = final_pass ? 1 : 0;
    OneVolumeYx &sc = p.sched;
    sc.mask = mask;
    sc.out_u16 = out_u16;
    sc.field_out = field_out;
    sc.nz = nz;
    sc.ny = ny;
    sc.nx = nx;
    sc.rows_yzx = out_rows ? 1 : 0;
    sc.n_ty = (int) ceil_div(ny, kTM);
    sc.n_tx = (int) ceil_div(nx, kXTN);
    sc.n_tiles = nz * sc.n_ty * sc.n_tx;
    sc.magic_tx = yx_div_magic((uint32_t) sc.n_tx);
    sc.magic_ty = yx_div_magic((uint32_t) sc.n_ty);

    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) ny, (cuuint64_t) nz};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * ny * 2)};
    const cuuint32_t box[3] = {64u, (cuuint32_t) p.t.kp, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = tc_encode_fn()(&map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                                 const_cast<S *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    // Store map of the next field (not final): 32 x-voxels x 32 rows per store,
    // 64-byte swizzle; [y][z][x] rows as (x, z, y) from the window's first plane.
    CUtensorMap omap = map;
    if (!final_pass) {
        const cuuint32_t zbox[3] = {32u, 32u, 1u}, rbox[3] = {32u, 1u, 32u};
        const cuuint64_t rdims[3] = {(cuuint64_t) nx, (cuuint64_t) nz, (cuuint64_t) ny};
        const cuuint64_t rstrides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (out_rows ? out_rows->nz_total * nx * 2 : 0)};
        void *obase = out_rows ? static_cast<void *>(static_cast<S *>(out_rows->base) + out_rows->z0 * nx)
                               : static_cast<void *>(out);
        cr = tc_encode_fn()(&omap, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                            obase, out_rows ? rdims : dims, out_rows ? rstrides : strides, out_rows ? rbox : zbox,
                            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                            CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    }
    int dev = 0, sms = 148, smem_max = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    p.stages = yx_stages(p.t.kp, p.t.kpa, smem_max);
    const int smem = yx_smem_bytes(p.t.kp, p.t.kpa, p.stages);
    if (smem > smem_max) return cudaErrorInvalidValue;
    auto *kern = mask_fmt == MAXI_MASK_U8
                     ? (final_pass ? tc_yx_kernel<S, MAXI_MASK_U8, true, OneVolumeYx>
                                   : tc_yx_kernel<S, MAXI_MASK_U8, false, OneVolumeYx>)
                     : (final_pass ? tc_yx_kernel<S, MAXI_MASK_BITPACKED, true, OneVolumeYx>
                                   : tc_yx_kernel<S, MAXI_MASK_BITPACKED, false, OneVolumeYx>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const int64_t grid = std::min<int64_t>(sc.n_tiles, sms);
    kern<<<(unsigned) grid, kYxThreads, smem, st>>>(map, omap, p);
    return cudaGetLastError();
}

template cudaError_t tc_yx<__nv_bfloat16>(const __nv_bfloat16 *, __nv_bfloat16 *, const void *, int, bool, uint16_t *,
                                          float *, int64_t, int64_t, int64_t, const float *, int, bool, bool,
                                          cudaStream_t, const YzRows *);
template cudaError_t tc_yx<__half>(const __half *, __half *, const void *, int, bool, uint16_t *, float *, int64_t,
                                   int64_t, int64_t, const float *, int, bool, bool, cudaStream_t, const YzRows *);

// The x pass in its transposed form (radius above kTcMaxRadius).
template <typename S>
static cudaError_t tc_contig_t(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass,
                               uint16_t *out_u16, float *field_out, int64_t nz, int64_t ny, int64_t nx,
                               const float *kernel, int radius, bool error_feedback, cudaStream_t st,
                               const YzRows *out_rows, bool hi_only) {
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    ContigLaunch<OneVolumeContigT> p{};
    const int ra = (int) round_up(radius, 8);
    fill_pass_taps(p.taps, kernel, radius, ra, (int) round_up(kXTN + ra + radius, 16), is_bf16, error_feedback,
                   hi_only);
    if (kXtRows * 2 + 2 * p.taps.kcols > (int) kTmemColsStrided) return cudaErrorInvalidValue;
    p.final_pass = final_pass ? 1 : 0;
    OneVolumeContigT &sc = p.sched;
    sc.out = out_rows ? out_rows->base : out;
    sc.mask = mask;
    sc.out_u16 = out_u16;
    sc.field_out = field_out;
    sc.rows = nz * ny;
    sc.nx = nx;
    sc.ny = ny;
    sc.out_nz = out_rows ? out_rows->nz_total : 0;
    sc.out_z0 = out_rows ? out_rows->z0 : 0;
    sc.n_xt = (int) ceil_div(nx, kXTN);
    sc.n_tiles = (int64_t) sc.n_xt * ceil_div(sc.rows, kXtRows);

    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) sc.rows, 1};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * sc.rows * 2)};
    const cuuint32_t box[3] = {64u, (cuuint32_t) kXtRows, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = tc_encode_fn()(&map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                                 const_cast<S *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const int smem = contig_t_smem_bytes(p.taps.kpa);
    auto *kern = mask_fmt == MAXI_MASK_U8 ? tc_contig_t_kernel<S, MAXI_MASK_U8> : tc_contig_t_kernel<S, MAXI_MASK_BITPACKED>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(sc.n_tiles, sms);
    kern<<<(unsigned) grid, kXtThreads, smem, st>>>(map, p);
    return cudaGetLastError();
}

template <typename S>
cudaError_t tc_contig(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass, uint16_t *out_u16,
                      float *field_out, int64_t nz, int64_t ny, int64_t nx, const float *kernel, int radius,
                      bool error_feedback, cudaStream_t st, const YzRows *out_rows, bool hi_only) {
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    if (final_pass) out_rows = nullptr;
    if (radius > kTcMaxRadius)
        return tc_contig_t<S>(in, out, mask, mask_fmt, final_pass, out_u16, field_out, nz, ny, nx, kernel, radius,
                              error_feedback, st, out_rows, hi_only);
    ContigLaunch<OneVolumeContig> p{};
    const int ra = (int) round_up(radius, 8);
    fill_pass_taps(p.taps, kernel, radius, ra, (int) round_up(kXTN + ra + radius, 16), is_bf16, error_feedback,
                   hi_only);
    p.final_pass = final_pass ? 1 : 0;
    OneVolumeContig &sc = p.sched;
    sc.out = out_rows ? out_rows->base : out;
    sc.mask = mask;
    sc.out_u16 = out_u16;
    sc.field_out = field_out;
    sc.rows = nz * ny;
    sc.nx = nx;
    sc.ny = ny;
    sc.out_nz = out_rows ? out_rows->nz_total : 0;
    sc.out_z0 = out_rows ? out_rows->z0 : 0;
    sc.n_xt = (int) ceil_div(nx, kXTN);
    sc.n_tiles = (int64_t) sc.n_xt * ceil_div(sc.rows, kTM);

    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) sc.rows, 1};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * sc.rows * 2)};
    const cuuint32_t box[3] = {64u, (cuuint32_t) kTM, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = tc_encode_fn()(&map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                                 const_cast<S *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                                 CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const int smem = contig_smem_bytes_tc(p.taps.kp, p.taps.kpa);
    auto *kern = mask_fmt == MAXI_MASK_U8 ? tc_contig_kernel<S, MAXI_MASK_U8, OneVolumeContig>
                                          : tc_contig_kernel<S, MAXI_MASK_BITPACKED, OneVolumeContig>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(sc.n_tiles, sms);
    kern<<<(unsigned) grid, kXThreads, smem, st>>>(map, p);
    return cudaGetLastError();
}

template cudaError_t tc_contig<__nv_bfloat16>(const __nv_bfloat16 *, __nv_bfloat16 *, const void *, int, bool,
                                              uint16_t *, float *, int64_t, int64_t, int64_t, const float *, int,
                                              bool, cudaStream_t, const YzRows *, bool);
template cudaError_t tc_contig<__half>(const __half *, __half *, const void *, int, bool, uint16_t *, float *,
                                       int64_t, int64_t, int64_t, const float *, int, bool, cudaStream_t,
                                       const YzRows *, bool);

int tc_read_and_clear_error() {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_tc_error, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return -1;
    }
    if (v != 0) {
        const int zero = 0;
        cudaMemcpyToSymbol(g_tc_error, &zero, sizeof(int));
    }
    return v;
}

}  // namespace tc
}  // namespace maxi
