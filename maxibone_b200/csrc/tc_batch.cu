// Multi-volume tensor-core passes: one persistent launch per pass covers the
// tiles of every volume of a group (volumes with the same kernel and
// repetition count), so a batch of small and uneven volumes fills all SMs
// instead of one under-filled launch per volume.
//
// The per-volume data -- tensor maps of both ping-pong buffers for each pass,
// pointers, shape and tile counts -- live in a device table; a CTA walks the
// batch's global column (z/y) or tile (x) index, finds its volume with a
// binary search over the prefix sums, and then works exactly like the
// single-volume kernels in tc_pass.cu (same Toeplitz operands, pipeline,
// bounded waits and epilogues).
#include <cudaTypedefs.h>

#include "host_util.h"
#include "tc_kernels.cuh"
#include "tc_yx.cuh"

namespace maxi {
namespace tc {

TcGeometry tc_geometry(int radius) {
    TcGeometry g;
    g.radius = radius;
    g.kp_strided = (int) round_up(kTM + 2 * radius, 16);
    g.kpa_strided = (int) round_up(g.kp_strided, 64);
    g.ra = (int) round_up(radius, 8);
    g.kp_contig = (int) round_up(kXTN + g.ra + radius, 16);
    g.kpa_contig = (int) round_up(g.kp_contig, 64);
    return g;
}

// Fills the tile counts and the ten tensor maps of one volume.
int tc_fill_volume(TcVol &vol, void *buf0, void *buf1, const uint32_t *packed_mask, uint16_t *out_u16,
                   float *field_out, int64_t nz, int64_t ny, int64_t nx, bool is_bf16, const TcGeometry &g) {
    vol = TcVol{};
    vol.buf[0] = buf0;
    vol.buf[1] = buf1;
    vol.mask = packed_mask;
    vol.out_u16 = out_u16;
    vol.field_out = field_out;
    vol.nz = nz; vol.ny = ny; vol.nx = nx;
    vol.n_at_z = (int) ceil_div(nz, kTM);
    vol.n_at_y = (int) ceil_div(ny, kTM);
    vol.n_xc_z = (int) ceil_div(nx, StridedShape<true>::kTN);
    vol.n_xc_y = (int) ceil_div(nx, StridedShape<false>::kTN);
    vol.n_xt = (int) ceil_div(nx, kXTN);
    vol.cols_z = (int64_t) vol.n_xc_z * ny;
    vol.cols_y = (int64_t) vol.n_xc_y * nz;
    vol.tiles_x = (int64_t) vol.n_xt * ceil_div(nz * ny, kTM);
    vol.tiles_yx = (int64_t) vol.n_xt * vol.n_at_y * nz;
    vol.magic_xt = yx_div_magic((uint32_t) vol.n_xt);
    vol.magic_at_y = yx_div_magic((uint32_t) vol.n_at_y);
    auto enc = tc_encode_fn();
    if (!enc) return -1;
    const CUtensorMapDataType dt = is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    const cuuint32_t estr[3] = {1, 1, 1};
    for (int b = 0; b < 2; b++) {
        void *base = vol.buf[b];
        const cuuint64_t d3[3] = {(cuuint64_t) nx, (cuuint64_t) ny, (cuuint64_t) nz};
        const cuuint64_t s3[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * ny * 2)};
        const cuuint32_t boxz[3] = {64u, 1u, (cuuint32_t) g.kp_strided};
        const cuuint32_t boxy[3] = {64u, (cuuint32_t) g.kp_strided, 1u};
        const cuuint64_t dx[3] = {(cuuint64_t) nx, (cuuint64_t) (nz * ny), 1};
        const cuuint64_t sx[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * nz * ny * 2)};
        const cuuint32_t boxx[3] = {64u, (cuuint32_t) kTM, 1u};
        const cuuint32_t boxs[3] = {32u, 32u, 1u};
        const cuuint64_t dr[3] = {(cuuint64_t) nx, (cuuint64_t) nz, (cuuint64_t) ny};
        const cuuint64_t sr[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nz * nx * 2)};
        const cuuint32_t boxr[3] = {64u, (cuuint32_t) g.kp_strided, 1u};
        const cuuint32_t boxyx[3] = {32u, 1u, 32u};
        if (enc(&vol.map[0][b], dt, 3, base, d3, s3, boxz, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.map[1][b], dt, 3, base, d3, s3, boxy, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.map[2][b], dt, 3, base, dx, sx, boxx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.ystore[b], dt, 3, base, d3, s3, boxs, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.zrows[b], dt, 3, base, dr, sr, boxr, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.yxrows[b], dt, 3, base, dr, sr, boxyx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return -1;
    }
    return 0;
}

cudaError_t tc_batch_pass(const TcVol *d_vols, const int64_t *d_prefix, int64_t total, int n_vol, int pass, int in_buf,
                          bool final_pass, const float *kernel, const TcGeometry &g, bool is_bf16, bool error_feedback,
                          bool rows_yz, cudaStream_t st, bool hi_only) {
    if (total == 0) return cudaSuccess;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned) std::min<int64_t>(total, sms);
    CUtensorMap unused{};  // the batch kernels read their maps from the volume table
    cudaError_t e;
    if (pass == 3) {
        if (!hi_only || g.radius > kTcMaxRadius || g.kp_contig != g.kp_strided) return cudaErrorInvalidValue;
        YxLaunch<ManyVolumesYx> p{};
        fill_pass_taps(p.t, kernel, g.radius, g.ra, g.kp_contig, is_bf16, error_feedback, true);
        p.final_pass = final_pass ? 1 : 0;
        int smem_max = 0;
        cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
        p.stages = yx_stages(p.t.kp, p.t.kpa, smem_max);
        p.sched.vols = d_vols;
        p.sched.prefix = d_prefix;
        p.sched.n_vol = n_vol;
        p.sched.in_buf = in_buf;
        const int smem = yx_smem_bytes(p.t.kp, p.t.kpa, p.stages);
        if (smem > smem_max) return cudaErrorInvalidValue;
        auto *k = is_bf16 ? (final_pass ? tc_yx_kernel<__nv_bfloat16, MAXI_MASK_BITPACKED, true, ManyVolumesYx>
                                        : tc_yx_kernel<__nv_bfloat16, MAXI_MASK_BITPACKED, false, ManyVolumesYx>)
                          : (final_pass ? tc_yx_kernel<__half, MAXI_MASK_BITPACKED, true, ManyVolumesYx>
                                        : tc_yx_kernel<__half, MAXI_MASK_BITPACKED, false, ManyVolumesYx>);
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
        k<<<grid, kYxThreads, smem, st>>>(unused, unused, p);
    } else if (pass == 2) {
        ContigLaunch<ManyVolumesContig> p{};
        fill_pass_taps(p.taps, kernel, g.radius, g.ra, g.kp_contig, is_bf16, error_feedback, hi_only);
        p.final_pass = final_pass ? 1 : 0;
        p.sched.vols = d_vols;
        p.sched.prefix = d_prefix;
        p.sched.n_vol = n_vol;
        p.sched.in_buf = in_buf;
        p.sched.out_rows = (rows_yz && !final_pass) ? 1 : 0;
        const int smem = contig_smem_bytes_tc(p.taps.kp, p.taps.kpa);
        auto *k = is_bf16 ? tc_contig_kernel<__nv_bfloat16, MAXI_MASK_BITPACKED, ManyVolumesContig>
                          : tc_contig_kernel<__half, MAXI_MASK_BITPACKED, ManyVolumesContig>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
        k<<<grid, kXThreads, smem, st>>>(unused, p);
    } else {
        const bool axis_z = pass == 0;
        StridedLaunch<ManyVolumesStrided> p{};
        fill_pass_taps(p.taps, kernel, g.radius, 0, g.kp_strided, is_bf16, error_feedback, hi_only);
        p.sched.vols = d_vols;
        p.sched.prefix = d_prefix;
        p.sched.n_vol = n_vol;
        p.sched.axis_z = axis_z ? 1 : 0;
        p.sched.in_buf = in_buf;
        p.sched.z_in_rows = (axis_z && rows_yz) ? 1 : 0;
        p.sched.tn = axis_z ? StridedShape<true>::kTN : StridedShape<false>::kTN;
        const int smem = strided_smem_bytes(p.taps.kp, p.sched.tn,
                                            axis_z ? StridedShape<true>::kStages : StridedShape<false>::kStages);
        auto *k = axis_z ? (is_bf16 ? tc_strided_kernel<__nv_bfloat16, true, 128, ManyVolumesStrided>
                                    : tc_strided_kernel<__half, true, 128, ManyVolumesStrided>)
                         : (is_bf16 ? tc_strided_kernel<__nv_bfloat16, false, 128, ManyVolumesStrided>
                                    : tc_strided_kernel<__half, false, 128, ManyVolumesStrided>);
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
        k<<<grid, kThreads, smem, st>>>(unused, unused, p);
    }
    return cudaGetLastError();
}

int tc_batch_read_and_clear_error() {
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
