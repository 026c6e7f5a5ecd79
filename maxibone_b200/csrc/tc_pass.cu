// Single-volume tensor-core passes for 16-bit field storage (BF16 / FP16):
// host side of the kernels in tc_kernels.cuh (tensor maps with the volume's
// shape, one persistent launch per pass, one CTA per SM).
#include <cudaTypedefs.h>

#include <mutex>

#include "host_util.h"
#include "profiler.h"
#include "tc_kernels.cuh"

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
                       int radius, bool error_feedback, cudaStream_t st, const YzRows *in_rows) {
    if (!axis_z) in_rows = nullptr;
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    const int tn = strided_tn(radius), stages = kStridedStages;
    StridedLaunch<OneVolumeStrided> p{};
    fill_pass_taps(p.taps, kernel, radius, 0, (int) round_up(kTM + 2 * radius, 16), is_bf16, error_feedback);
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
                                               bool, const float *, int, bool, cudaStream_t, const YzRows *);
template cudaError_t tc_strided<__half>(const __half *, __half *, int64_t, int64_t, int64_t, bool, const float *, int,
                                        bool, cudaStream_t, const YzRows *);

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

// The x pass in its transposed form (radius above kTcMaxRadius).
template <typename S>
static cudaError_t tc_contig_t(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass,
                               uint16_t *out_u16, float *field_out, int64_t nz, int64_t ny, int64_t nx,
                               const float *kernel, int radius, bool error_feedback, cudaStream_t st,
                               const YzRows *out_rows) {
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    ContigLaunch<OneVolumeContigT> p{};
    const int ra = (int) round_up(radius, 8);
    fill_pass_taps(p.taps, kernel, radius, ra, (int) round_up(kXTN + ra + radius, 16), is_bf16, error_feedback);
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
                      bool error_feedback, cudaStream_t st, const YzRows *out_rows) {
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    if (final_pass) out_rows = nullptr;
    if (radius > kTcMaxRadius)
        return tc_contig_t<S>(in, out, mask, mask_fmt, final_pass, out_u16, field_out, nz, ny, nx, kernel, radius,
                              error_feedback, st, out_rows);
    ContigLaunch<OneVolumeContig> p{};
    const int ra = (int) round_up(radius, 8);
    fill_pass_taps(p.taps, kernel, radius, ra, (int) round_up(kXTN + ra + radius, 16), is_bf16, error_feedback);
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
                                              bool, cudaStream_t, const YzRows *);
template cudaError_t tc_contig<__half>(const __half *, __half *, const void *, int, bool, uint16_t *, float *,
                                       int64_t, int64_t, int64_t, const float *, int, bool, cudaStream_t,
                                       const YzRows *);

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
