// Tensor-core (tcgen05) z and y passes for 16-bit field storage (BF16 / FP16).
//
// A 1-D convolution along an axis is a banded Toeplitz matrix product.  For a
// tile of 128 consecutive outputs along the axis and 128 x-columns:
//
//     D[o, x] = sum_j T[o, j] * F[a0 - R + j, x],   T[o, j] = k[j - o] for 0 <= j - o <= 2R
//
// M = 128 outputs (TMEM lanes), N = 128 x-columns (TMEM columns), K = KP >=
// 128 + 2R input rows.  T is built once per CTA in shared memory (K-major,
// 128-byte swizzle); the field tile F arrives by TMA (x contiguous: MN-major,
// 128-byte swizzle; rows outside the volume are zero-filled by TMA, which is
// exactly the reference's zero boundary).  Coefficients are split into a high
// and a low 16-bit part (T = T_hi + T_lo, two MMAs into one FP32 accumulator)
// so the effective kernel keeps ~16 significant bits and its sum stays 1 to
// ~1e-6: with single-rounded 16-bit coefficients the kernel's gain error
// compounds over 3 x R passes.  FP16 coefficients are scaled by 2^10 to stay in
// the normal range; the epilogue undoes the scale exactly.
//
// Warp roles in a persistent CTA (one per SM): warp 0 issues TMA loads into a
// 2-stage ring, warp 1 issues the MMAs (one thread) into a double-buffered TMEM
// accumulator, warps 2-5 drain TMEM (tcgen05.ld), narrow to the storage type
// and store.  With error feedback on, the rounding error of each stored value
// is carried to its x-neighbour (32-voxel chains along x): the stored field's
// rounding noise becomes high-pass along x and the next x pass removes it.
#include <cudaTypedefs.h>

#include <mutex>

#include "host_util.h"
#include "profiler.h"
#include "tc_common.cuh"
#include "tc_pass.h"
#include "tc_batch.h"

namespace maxi {
namespace tc {

constexpr int kTM = 128;      // outputs along the axis per tile
constexpr int kTN = 128;      // x columns per tile
constexpr int kStages = 2;    // TMA ring depth (x pass)

constexpr int kPrefetch = 3;  // tiles prefetched into L2 ahead of the ring
constexpr int kEpiWarps = 8;  // two warps per TMEM lane quadrant, each drains half the columns
constexpr int kThreads = 64 + 32 * kEpiWarps;  // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue

struct StridedParams {
    void *out;
    int64_t A;          // axis length
    int64_t n_other;    // the third coordinate (y for the z pass, z for the y pass)
    int64_t nx;
    int64_t stride_a;   // element stride along the axis in `out`
    int64_t stride_o;   // element stride of the third coordinate
    int n_at, n_xc;     // axis tiles, x chunks
    int64_t n_cols;     // columns = x chunks x third coordinate; a CTA marches a column's axis tiles
    int radius, kp, kpa; // radius, K (multiple of 16), K rounded to 64
    int axis_is_z;
    float inv_scale;
    int error_feedback;
    uint16_t hi[2 * kTcMaxRadius + 1];
    uint16_t lo[2 * kTcMaxRadius + 1];
};

// Per-epilogue-warp staging of a 32-row x 32-column output chunk: row stride
// 80 bytes (16-byte stores of 32 lanes on 32 rows hit 8 distinct bank groups).
constexpr int kStageWarpBytes = 2 * 32 * 64;  // two 32 x 32 16-bit buffers per epilogue warp

__host__ __device__ constexpr int strided_smem_bytes(int kp, int kpa, int tn, int stages) {
    return 1024 /*alignment slack*/ + 2 * kpa * kTM * 2 /*T_hi, T_lo*/ + stages * (tn / 64) * kp * 128 /*B ring*/ +
           1024 /*barriers, TMEM slot*/ + kEpiWarps * kStageWarpBytes;
}

// TN x-columns per tile, STAGES-deep TMA ring.  The z pass uses 128-column tiles
// (256 contiguous bytes per plane row per tile) and stages its stores so one
// instruction writes 8 rows; the y pass uses 64-column tiles with a 4-deep ring
// and TMA bulk stores of each warp's 32 x 32 chunk.
template <typename S, int TN, int STAGES>
__global__ void __launch_bounds__(kThreads, 1)
tc_strided_pass(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmap_out,
                const __grid_constant__ StridedParams p) {
    constexpr int kStrTN = TN, kStrStages = STAGES, kStrChunks = TN / 64;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *t_hi = smem;
    uint8_t *t_lo = t_hi + p.kpa * kTM * 2;
    uint8_t *ring = t_lo + p.kpa * kTM * 2;
    const int stage_bytes = (kStrTN / 64) * p.kp * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kStrStages * stage_bytes);
    uint64_t *full = bars, *empty = bars + kStrStages, *tfull = bars + 2 * kStrStages, *tempty = bars + 2 * kStrStages + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStrStages + 4);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;  // 1024-byte aligned

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // Toeplitz operands, K-major with 128-byte swizzle, zero outside the band.
    for (int e = threadIdx.x; e < kTM * p.kpa; e += kThreads) {
        const int o = e / p.kpa, k = e - o * p.kpa;
        const int t = k - o;
        uint16_t h = 0, l = 0;
        if (t >= 0 && t <= 2 * p.radius && k < p.kp) { h = p.hi[t]; l = p.lo[t]; }
        const uint32_t off = sw128_kmajor_offset(o, k, kTM);
        *reinterpret_cast<uint16_t *>(t_hi + off) = h;
        *reinterpret_cast<uint16_t *>(t_lo + off) = l;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStrStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kEpiWarps); }
        fence_barrier_init();
        prefetch_tmap(&tmap);
    }
    __syncwarp();
    if (warp == 0) {
        tmem_alloc(tmem_slot, 2 * kStrTN);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        // TMA producer.
        int64_t tl = 0;
        bool ok = true;
        for (int64_t col = blockIdx.x; ok && col < p.n_cols; col += gridDim.x)
        for (int at = 0; at < p.n_at; at++, tl++) {
            const int s = (int) (tl % kStrStages);
            const uint32_t ph = (uint32_t) ((tl / kStrStages) & 1);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) { ok = false; break; }
            {
                // L2 prefetch of the tile kPrefetch tiles ahead in this CTA's order.
                const int64_t tp = tl + kPrefetch;
                const int64_t colp = blockIdx.x + (tp / p.n_at) * gridDim.x;
                if (colp < p.n_cols) {
                    const int atp = (int) (tp % p.n_at);
                    const int xcp = (int) (colp % p.n_xc), othp = (int) (colp / p.n_xc);
                    for (int c = 0; c < kStrTN / 64; c++) {
                        if (p.axis_is_z) tma_prefetch_3d(&tmap, xcp * kStrTN + 64 * c, othp, atp * kTM - p.radius);
                        else tma_prefetch_3d(&tmap, xcp * kStrTN + 64 * c, atp * kTM - p.radius, othp);
                    }
                }
            }
            const int xc = (int) (col % p.n_xc);
            const int oth = (int) (col / p.n_xc);
            const int a_in = at * kTM - p.radius;
            const int x0 = xc * kStrTN;
            mbar_arrive_expect_tx(&full[s], stage_bytes);
            for (int c = 0; c < kStrTN / 64; c++) {
                uint8_t *dst = ring + s * stage_bytes + c * p.kp * 128;
                if (p.axis_is_z) tma_load_3d(dst, &tmap, x0 + 64 * c, oth, a_in, &full[s]);
                else tma_load_3d(dst, &tmap, x0 + 64 * c, a_in, oth, &full[s]);
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc = idesc_f16(fmt, 0 /*A K-major*/, 1 /*B MN-major*/, kTM, kStrTN);
        const uint32_t a_hi = smem_u32(t_hi), a_lo = smem_u32(t_lo), b0 = smem_u32(ring);
        int64_t tl = 0;
        bool ok = true;
        for (int64_t col = blockIdx.x; ok && col < p.n_cols; col += gridDim.x)
        for (int at = 0; at < p.n_at; at++, tl++) {
            const int s = (int) (tl % kStrStages);
            const uint32_t ph = (uint32_t) ((tl / kStrStages) & 1);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&full[s], ph, 1) || !mbar_wait(&tempty[d], dph ^ 1, 3)) { ok = false; break; }
            tc_fence_after();
            const uint32_t dt = tmem + d * kStrTN;
            for (int ks = 0; ks < p.kp / 16; ks++) {
                const uint32_t koff = (ks >> 2) * (kTM * 128) + (ks & 3) * 32;
                const uint64_t bd = smem_desc_sw128(b0 + s * stage_bytes + ks * 2048, p.kp * 128, 1024);
                umma_f16(dt, smem_desc_sw128(a_hi + koff, 16, 1024), bd, idesc, ks > 0 ? 1u : 0u);
                umma_f16(dt, smem_desc_sw128(a_lo + koff, 16, 1024), bd, idesc, 1u);
            }
            umma_commit(&empty[s]);
            umma_commit(&tfull[d]);
        }
    } else if (warp >= 2) {
        // Epilogue: TMEM -> registers -> storage type -> global.
        const int quad = warp & 3;           // TMEM lane quadrant this warp may access
        const int half = (warp - 2) >> 2;    // which half of the columns it drains
        const int o = quad * 32 + lane;      // output row within the tile
        S *out = static_cast<S *>(p.out);
        uint8_t *stg = stage_out + (warp - 2) * kStageWarpBytes;  // two 32 x 32 staging buffers
        int sbuf = 0;
        int64_t tl = 0;
        bool ok = true;
        for (int64_t col = blockIdx.x; ok && col < p.n_cols; col += gridDim.x)
        for (int at = 0; at < p.n_at; at++, tl++) {
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&tfull[d], dph, 2)) { ok = false; break; }
            tc_fence_after();
            const int xc = (int) (col % p.n_xc);
            const int64_t oth = col / p.n_xc;
            const int64_t x0 = (int64_t) xc * kStrTN;
            const int c0 = half * kStrChunks;  // this warp's 32-column chunks
            const uint32_t tbase = tmem + ((uint32_t) (quad * 32) << 16) + d * kStrTN;
#pragma unroll
            for (int cc = 0; cc < kStrChunks; cc++) {
                float va[32];
                __syncwarp();
                tmem_ld32(tbase + (c0 + cc) * 32, va);
                uint16_t q[32];
                narrow32<S>(va, p.inv_scale, p.error_feedback, q);
                const int64_t xb = x0 + (c0 + cc) * 32;
                if (p.axis_is_z) {
                    // z pass: lanes' rows lie on different planes (2 MB apart at 1024^2);
                    // stage the 32 x 32 chunk and write 8 rows (8 x 64 bytes) per instruction.
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 4; i++) *reinterpret_cast<uint4 *>(stg + lane * 80 + i * 16) = pack8(q + 8 * i);
                    __syncwarp();
                    const int sub = lane & 3, rsub = lane >> 2;
#pragma unroll
                    for (int r4 = 0; r4 < 4; r4++) {
                        const int rr = r4 * 8 + rsub;
                        const int64_t ar = (int64_t) at * kTM + quad * 32 + rr;
                        const uint4 w = *reinterpret_cast<const uint4 *>(stg + rr * 80 + sub * 16);
                        if (ar < p.A && xb + sub * 8 < p.nx)
                            *reinterpret_cast<uint4 *>(out + ar * p.stride_a + oth * p.stride_o + xb + sub * 8) = w;
                    }
                    continue;
                }
                // y pass: TMA store of the warp's 32 rows x 32 columns (64-byte swizzle of
                // the store tensor map) instead of 32 per-lane row stores.
                if (lane == 0) bulk_wait_read<1>();  // the store issued two chunks ago has read this buffer
                __syncwarp();
                uint8_t *sb = stg + sbuf * 2048;
#pragma unroll
                for (int i = 0; i < 4; i++)
                    *reinterpret_cast<uint4 *>(sb + lane * 64 + ((i ^ ((lane >> 1) & 3)) << 4)) = pack8(q + 8 * i);
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    tma_store_3d(&tmap_out, sb, (int) xb, at * kTM + quad * 32, (int) oth);
                    bulk_commit();
                }
                sbuf ^= 1;
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[d]);
        }
    }
    if (warp >= 2 && lane == 0) bulk_wait_all();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * kStrTN);
    }
}

// ---- x pass -----------------------------------------------------------------------
//
// The x pass with the field as the A operand: 128 volume rows (M, TMEM lanes)
// x 128 x-outputs, so each epilogue thread owns 32 consecutive voxels of one
// row -- the layout re-illumination, error feedback along x and vector stores
// want.  D[r, o] = sum_j F[r, x0 - RA + j] * Tt[j, o] with RA = R rounded up to
// 8 (TMA x coordinates must be 16-byte aligned); Tt[j, o] = k[j - o - RA + R].
// The high and low coefficient halves sit in one K-major operand (rows
// 0..127 Tt_hi, 128..255 Tt_lo); two N = 128 MMAs accumulate both into the
// same FP32 accumulator, so the epilogue reads one value per voxel.
constexpr int kXTN = 128;            // x outputs per tile
constexpr int kXThreads = kThreads;

struct ContigParams {
    void *out;             // storage-type field (not FINAL)
    const void *mask;
    uint16_t *out_u16;     // FINAL
    float *field_out;      // FINAL, optional
    int64_t rows, nx;
    int n_xt;              // x tiles
    int64_t n_tiles;
    int radius, ra, kp, kpa;
    int mask_fmt, final_pass, error_feedback;
    float inv_scale;
    uint16_t hi[2 * kTcMaxRadius + 1];
    uint16_t lo[2 * kTcMaxRadius + 1];
};

__host__ __device__ constexpr int contig_smem_bytes_tc(int kp, int kpa) {
    return 1024 + kpa * 2 * kXTN * 2 /*Tt_hi|Tt_lo, 256 rows*/ + kStages * (kpa / 64) * kTM * 128 /*A ring*/ + 256;
}

template <typename S, int FMT>
__global__ void __launch_bounds__(kXThreads, 1)
tc_contig_pass(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ ContigParams p) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *tt = smem;                                  // K-major, 256 rows (hi 0..127, lo 128..255)
    uint8_t *ring = tt + p.kpa * 2 * kXTN * 2;
    const int nkb = p.kpa / 64;                          // 64-wide x boxes per stage
    const int stage_bytes = nkb * kTM * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kStages * stage_bytes);
    uint64_t *full = bars, *empty = bars + kStages, *tfull = bars + 2 * kStages, *tempty = bars + 2 * kStages + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    for (int e = threadIdx.x; e < 2 * kXTN * p.kpa; e += kXThreads) {
        const int n = e / p.kpa, j = e - n * p.kpa;
        const int o = n & (kXTN - 1);
        const int t = j - o - p.ra + p.radius;  // tap index 0..2R
        uint16_t v = 0;
        if (t >= 0 && t <= 2 * p.radius && j < p.kp) v = n < kXTN ? p.hi[t] : p.lo[t];
        *reinterpret_cast<uint16_t *>(tt + sw128_kmajor_offset(n, j, 2 * kXTN)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kEpiWarps); }
        fence_barrier_init();
        prefetch_tmap(&tmap);
    }
    __syncwarp();
    if (warp == 0) {
        tmem_alloc(tmem_slot, 2 * kXTN);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        int64_t tl = 0;
        for (int64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x, tl++) {
            const int s = (int) (tl % kStages);
            const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) break;
            const int64_t tp = tile + kPrefetch * (int64_t) gridDim.x;
            if (tp < p.n_tiles) {
                const int xsp = (int) (tp % p.n_xt) * kXTN - p.ra, r0p = (int) (tp / p.n_xt) * kTM;
                for (int kb = 0; kb < nkb; kb++) tma_prefetch_3d(&tmap, xsp + 64 * kb, r0p, 0);
            }
            const int xt = (int) (tile % p.n_xt);
            const int r0 = (int) (tile / p.n_xt) * kTM;
            const int xs = xt * kXTN - p.ra;
            mbar_arrive_expect_tx(&full[s], stage_bytes);
            for (int kb = 0; kb < nkb; kb++)
                tma_load_3d(ring + s * stage_bytes + kb * kTM * 128, &tmap, xs + 64 * kb, r0, 0, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc = idesc_f16(fmt, 0 /*A K-major*/, 0 /*B K-major*/, kTM, kXTN);
        const uint32_t a0 = smem_u32(ring), b0 = smem_u32(tt);
        int64_t tl = 0;
        for (int64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x, tl++) {
            const int s = (int) (tl % kStages);
            const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&full[s], ph, 1) || !mbar_wait(&tempty[d], dph ^ 1, 3)) break;
            tc_fence_after();
            const uint32_t dt = tmem + d * kXTN;
            for (int ks = 0; ks < p.kp / 16; ks++) {
                const uint32_t kin = (ks & 3) * 32;
                const uint64_t ad = smem_desc_sw128(a0 + s * stage_bytes + (ks >> 2) * (kTM * 128) + kin, 16, 1024);
                const uint32_t bhi = b0 + (ks >> 2) * (2 * kXTN * 128) + kin;  // rows 0..127: Tt_hi
                umma_f16(dt, ad, smem_desc_sw128(bhi, 16, 1024), idesc, ks > 0 ? 1u : 0u);
                umma_f16(dt, ad, smem_desc_sw128(bhi + kXTN * 128, 16, 1024), idesc, 1u);  // rows 128..255: Tt_lo
            }
            umma_commit(&empty[s]);
            umma_commit(&tfull[d]);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3;
        const int half = (warp - 2) >> 2;
        const int r = quad * 32 + lane;
        int64_t tl = 0;
        for (int64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x, tl++) {
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&tfull[d], dph, 2)) break;
            tc_fence_after();
            const int64_t row = (tile / p.n_xt) * kTM + r;
            const int64_t xa = (tile % p.n_xt) * kXTN + half * 64;  // this warp's 64 voxels of the row
            // Mask flags fetched before the TMEM loads.
            uint32_t mw[2];
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int64_t xb = xa + cc * 32;
                mw[cc] = (row < p.rows && xb < p.nx)
                             ? row_mask32<FMT>(p.mask, row * p.nx + xb, p.nx - xb < 32 ? (int) (p.nx - xb) : 32,
                                               p.rows * p.nx)
                             : 0u;
            }
            float ha[32], hb[32];
            __syncwarp();
            const uint32_t ta = tmem + ((uint32_t) (quad * 32) << 16) + d * kXTN + half * 64;
            tmem_ld32(ta, ha);
            tmem_ld32(ta + 32, hb);
            contig_epilogue64<S>(ha, hb, mw[0], mw[1], row, p.rows, p.nx, xa, p.inv_scale, p.error_feedback,
                                 p.final_pass, static_cast<uint16_t *>(p.out), p.out_u16, p.field_out);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[d]);
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * kXTN);
    }
}

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
    if (radius < 1 || radius > kTcMaxRadius) return false;
    if (nx % 8 != 0 || nx < 64) return false;  // TMA: 16-byte row strides, at least one 64-wide box
    if (nz > INT32_MAX / 2 || ny > INT32_MAX / 2 || nx > INT32_MAX / 2) return false;
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return major == 10 && tc_encode_fn() != nullptr;
}

template <typename S>
cudaError_t tc_strided(const S *in, S *out, int64_t nz, int64_t ny, int64_t nx, bool axis_z, const float *kernel,
                       int radius, bool error_feedback, cudaStream_t st) {
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    StridedParams p{};
    p.out = out;
    p.nx = nx;
    p.radius = radius;
    p.kp = (int) round_up(kTM + 2 * radius, 16);
    p.kpa = (int) round_up(p.kp, 64);
    p.axis_is_z = axis_z ? 1 : 0;
    p.error_feedback = error_feedback ? 1 : 0;
    const float scale = is_bf16 ? 1.0f : 1024.0f;
    p.inv_scale = 1.0f / scale;
    tc_split_taps(kernel, radius, is_bf16, scale, p.hi, p.lo);
    if (axis_z) { p.A = nz; p.n_other = ny; p.stride_a = ny * nx; p.stride_o = nx; }
    else { p.A = ny; p.n_other = nz; p.stride_a = nx; p.stride_o = ny * nx; }
    p.n_at = (int) ceil_div(p.A, kTM);
    p.n_xc = (int) ceil_div(nx, axis_z ? 128 : 64);
    p.n_cols = (int64_t) p.n_xc * p.n_other;

    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) ny, (cuuint64_t) nz};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * ny * 2)};
    const cuuint32_t box[3] = {64u, axis_z ? 1u : (cuuint32_t) p.kp, axis_z ? (cuuint32_t) p.kp : 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = tc_encode_fn()(&map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                              const_cast<S *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;

    CUtensorMap map_out;
    const cuuint64_t odims[3] = {(cuuint64_t) nx, (cuuint64_t) ny, (cuuint64_t) nz};
    const cuuint32_t obox[3] = {32u, axis_z ? 1u : 32u, axis_z ? 32u : 1u};
    cr = tc_encode_fn()(&map_out, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3, out,
                        odims, strides, obox, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                        CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const int tn = axis_z ? 128 : 64, stages = axis_z ? 2 : 4;
    const int smem = strided_smem_bytes(p.kp, p.kpa, tn, stages);
    auto *kern = axis_z ? tc_strided_pass<S, 128, 2> : tc_strided_pass<S, 64, 4>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(p.n_cols, sms);
    kern<<<(unsigned) grid, kThreads, smem, st>>>(map, map_out, p);
    return cudaGetLastError();
}

template cudaError_t tc_strided<__nv_bfloat16>(const __nv_bfloat16 *, __nv_bfloat16 *, int64_t, int64_t, int64_t,
                                               bool, const float *, int, bool, cudaStream_t);
template cudaError_t tc_strided<__half>(const __half *, __half *, int64_t, int64_t, int64_t, bool, const float *, int,
                                        bool, cudaStream_t);

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

template <typename S>
cudaError_t tc_contig(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass, uint16_t *out_u16,
                      float *field_out, int64_t nz, int64_t ny, int64_t nx, const float *kernel, int radius,
                      bool error_feedback, cudaStream_t st) {
    const bool is_bf16 = std::is_same<S, __nv_bfloat16>::value;
    ContigParams p{};
    p.out = out;
    p.mask = mask;
    p.out_u16 = out_u16;
    p.field_out = field_out;
    p.rows = nz * ny;
    p.nx = nx;
    p.radius = radius;
    p.ra = (int) round_up(radius, 8);
    p.kp = (int) round_up(kXTN + p.ra + radius, 16);
    p.kpa = (int) round_up(p.kp, 64);
    p.mask_fmt = mask_fmt;
    p.final_pass = final_pass ? 1 : 0;
    p.error_feedback = error_feedback ? 1 : 0;
    const float scale = is_bf16 ? 1.0f : 1024.0f;
    p.inv_scale = 1.0f / scale;
    tc_split_taps(kernel, radius, is_bf16, scale, p.hi, p.lo);
    p.n_xt = (int) ceil_div(nx, kXTN);
    p.n_tiles = (int64_t) p.n_xt * ceil_div(p.rows, kTM);

    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) p.rows, 1};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * p.rows * 2)};
    const cuuint32_t box[3] = {64u, (cuuint32_t) kTM, 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = tc_encode_fn()(&map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                              const_cast<S *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const int smem = contig_smem_bytes_tc(p.kp, p.kpa);
    auto *kern = mask_fmt == MAXI_MASK_U8 ? tc_contig_pass<S, MAXI_MASK_U8> : tc_contig_pass<S, MAXI_MASK_BITPACKED>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(p.n_tiles, sms);
    kern<<<(unsigned) grid, kXThreads, smem, st>>>(map, p);
    return cudaGetLastError();
}

template cudaError_t tc_contig<__nv_bfloat16>(const __nv_bfloat16 *, __nv_bfloat16 *, const void *, int, bool,
                                              uint16_t *, float *, int64_t, int64_t, int64_t, const float *, int,
                                              bool, cudaStream_t);
template cudaError_t tc_contig<__half>(const __half *, __half *, const void *, int, bool, uint16_t *, float *,
                                       int64_t, int64_t, int64_t, const float *, int, bool, cudaStream_t);

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
