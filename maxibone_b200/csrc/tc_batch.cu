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
#include "tc_batch.h"
#include "tc_common.cuh"

namespace maxi {
namespace tc {

namespace {
constexpr int kTM = 128, kTN = 128, kXTN = 128, kStages = 2, kEpiWarps = 8;
constexpr int kThreads = 64 + 32 * kEpiWarps;
constexpr int kStageRowBytes = 80, kStageWarpBytes = 32 * kStageRowBytes;
}  // namespace

struct BatchLaunch {
    const TcVol *vols;
    const int64_t *prefix;  // n_vol + 1 entries: columns (z / y passes) or tiles (x pass)
    int n_vol;
    int pass;               // 0 z, 1 y, 2 x
    int in_buf;             // which ping-pong buffer holds the pass input
    int final_pass;         // x pass of the last repetition
    int radius, ra, kp, kpa;
    int error_feedback;
    int is_bf16;
    float inv_scale;
    uint16_t hi[2 * kTcMaxRadius + 1];
    uint16_t lo[2 * kTcMaxRadius + 1];
};

__device__ __forceinline__ int find_volume(const int64_t *prefix, int n_vol, int64_t g) {
    int lo = 0, hi = n_vol - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// ---- z / y passes ---------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(kThreads, 1) tc_batch_strided(const __grid_constant__ BatchLaunch p) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *t_hi = smem;
    uint8_t *t_lo = t_hi + p.kpa * kTM * 2;
    uint8_t *ring = t_lo + p.kpa * kTM * 2;
    const int stage_bytes = (kTN / 64) * p.kp * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kStages * stage_bytes);
    uint64_t *full = bars, *empty = bars + kStages, *tfull = bars + 2 * kStages, *tempty = bars + 2 * kStages + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 4);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 256;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool is_z = p.pass == 0;
    const int64_t total = __ldg(p.prefix + p.n_vol);

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
        for (int s = 0; s < kStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kEpiWarps); }
        fence_barrier_init();
    }
    __syncwarp();
    if (warp == 0) {
        tmem_alloc(tmem_slot, 2 * kTN);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0 && lane == 0) {
        int64_t tl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x) {
            const int v = find_volume(p.prefix, p.n_vol, g);
            const TcVol &vol = p.vols[v];
            const int64_t col = g - __ldg(p.prefix + v);
            const int n_at = is_z ? vol.n_at_z : vol.n_at_y;
            const CUtensorMap *map = &vol.map[p.pass][p.in_buf];
            const int xc = (int) (col % vol.n_xc), oth = (int) (col / vol.n_xc);
            for (int at = 0; at < n_at; at++, tl++) {
                const int s = (int) (tl % kStages);
                const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
                if (!mbar_wait(&empty[s], ph ^ 1, 1)) { ok = false; break; }
                const int a_in = at * kTM - p.radius;
                mbar_arrive_expect_tx(&full[s], stage_bytes);
                for (int c = 0; c < kTN / 64; c++) {
                    uint8_t *dst = ring + s * stage_bytes + c * p.kp * 128;
                    if (is_z) tma_load_3d(dst, map, xc * kTN + 64 * c, oth, a_in, &full[s]);
                    else tma_load_3d(dst, map, xc * kTN + 64 * c, a_in, oth, &full[s]);
                }
            }
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_f16(p.is_bf16 ? 1u : 0u, 0, 1, kTM, kTN);
        const uint32_t a_hi = smem_u32(t_hi), a_lo = smem_u32(t_lo), b0 = smem_u32(ring);
        int64_t tl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x) {
            const int v = find_volume(p.prefix, p.n_vol, g);
            const int n_at = is_z ? p.vols[v].n_at_z : p.vols[v].n_at_y;
            for (int at = 0; at < n_at; at++, tl++) {
                const int s = (int) (tl % kStages);
                const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
                const int d = (int) (tl & 1);
                const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
                if (!mbar_wait(&full[s], ph, 1) || !mbar_wait(&tempty[d], dph ^ 1, 3)) { ok = false; break; }
                tc_fence_after();
                const uint32_t dt = tmem + d * kTN;
                for (int ks = 0; ks < p.kp / 16; ks++) {
                    const uint32_t koff = (ks >> 2) * (kTM * 128) + (ks & 3) * 32;
                    const uint64_t bd = smem_desc_sw128(b0 + s * stage_bytes + ks * 2048, p.kp * 128, 1024);
                    umma_f16(dt, smem_desc_sw128(a_hi + koff, 16, 1024), bd, idesc, ks > 0 ? 1u : 0u);
                    umma_f16(dt, smem_desc_sw128(a_lo + koff, 16, 1024), bd, idesc, 1u);
                }
                umma_commit(&empty[s]);
                umma_commit(&tfull[d]);
            }
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int o = quad * 32 + lane;
        uint8_t *stg = stage_out + (warp - 2) * kStageWarpBytes;
        int64_t tl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x) {
            const int v = find_volume(p.prefix, p.n_vol, g);
            const TcVol &vol = p.vols[v];
            const int64_t col = g - __ldg(p.prefix + v);
            const int n_at = is_z ? vol.n_at_z : vol.n_at_y;
            const int64_t A = is_z ? vol.nz : vol.ny;
            const int64_t stride_a = is_z ? vol.ny * vol.nx : vol.nx;
            const int64_t stride_o = is_z ? vol.nx : vol.ny * vol.nx;
            const int xc = (int) (col % vol.n_xc);
            const int64_t oth = col / vol.n_xc;
            S *out = static_cast<S *>(vol.buf[p.in_buf ^ 1]);
            for (int at = 0; at < n_at; at++, tl++) {
                const int d = (int) (tl & 1);
                const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
                if (!mbar_wait(&tfull[d], dph, 2)) { ok = false; break; }
                tc_fence_after();
                const int64_t a = (int64_t) at * kTM + o;
                const int64_t x0 = (int64_t) xc * kTN;
                const int c0 = half * 2;
                const uint32_t tbase = tmem + ((uint32_t) (quad * 32) << 16) + d * kTN;
#pragma unroll
                for (int cc = 0; cc < 2; cc++) {
                    float va[32];
                    __syncwarp();
                    tmem_ld32(tbase + (c0 + cc) * 32, va);
                    uint16_t q[32];
                    narrow32<S>(va, p.inv_scale, p.error_feedback, q);
                    const int64_t xb = x0 + (c0 + cc) * 32;
                    const uint4 u[4] = {pack8(q), pack8(q + 8), pack8(q + 16), pack8(q + 24)};
                    if (!is_z) {
                        if (a < A) {
                            S *dst = out + a * stride_a + oth * stride_o + xb;
#pragma unroll
                            for (int i = 0; i < 4; i++)
                                if (xb + 8 * i < vol.nx) reinterpret_cast<uint4 *>(dst)[i] = u[i];
                        }
                        continue;
                    }
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 4; i++) *reinterpret_cast<uint4 *>(stg + lane * kStageRowBytes + i * 16) = u[i];
                    __syncwarp();
                    const int sub = lane & 3, rsub = lane >> 2;
#pragma unroll
                    for (int r4 = 0; r4 < 4; r4++) {
                        const int rr = r4 * 8 + rsub;
                        const int64_t ar = (int64_t) at * kTM + quad * 32 + rr;
                        const uint4 w = *reinterpret_cast<const uint4 *>(stg + rr * kStageRowBytes + sub * 16);
                        if (ar < A && xb + sub * 8 < vol.nx)
                            *reinterpret_cast<uint4 *>(out + ar * stride_a + oth * stride_o + xb + sub * 8) = w;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[d]);
            }
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * kTN);
    }
}

// ---- x pass ---------------------------------------------------------------------
template <typename S>
__global__ void __launch_bounds__(kThreads, 1) tc_batch_contig(const __grid_constant__ BatchLaunch p) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *tt = smem;
    uint8_t *ring = tt + p.kpa * 2 * kXTN * 2;
    const int nkb = p.kpa / 64;
    const int stage_bytes = nkb * kTM * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kStages * stage_bytes);
    uint64_t *full = bars, *empty = bars + kStages, *tfull = bars + 2 * kStages, *tempty = bars + 2 * kStages + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kStages + 4);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = __ldg(p.prefix + p.n_vol);

    for (int e = threadIdx.x; e < 2 * kXTN * p.kpa; e += kThreads) {
        const int n = e / p.kpa, j = e - n * p.kpa;
        const int o = n & (kXTN - 1);
        const int t = j - o - p.ra + p.radius;
        uint16_t v = 0;
        if (t >= 0 && t <= 2 * p.radius && j < p.kp) v = n < kXTN ? p.hi[t] : p.lo[t];
        *reinterpret_cast<uint16_t *>(tt + sw128_kmajor_offset(n, j, 2 * kXTN)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kEpiWarps); }
        fence_barrier_init();
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
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int v = find_volume(p.prefix, p.n_vol, g);
            const TcVol &vol = p.vols[v];
            const int64_t tile = g - __ldg(p.prefix + v);
            const int s = (int) (tl % kStages);
            const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) break;
            const int xs = (int) (tile % vol.n_xt) * kXTN - p.ra;
            const int r0 = (int) (tile / vol.n_xt) * kTM;
            mbar_arrive_expect_tx(&full[s], stage_bytes);
            for (int kb = 0; kb < nkb; kb++)
                tma_load_3d(ring + s * stage_bytes + kb * kTM * 128, &vol.map[2][p.in_buf], xs + 64 * kb, r0, 0, &full[s]);
        }
    } else if (warp == 1 && lane == 0) {
        const uint32_t idesc = idesc_f16(p.is_bf16 ? 1u : 0u, 0, 0, kTM, kXTN);
        const uint32_t a0 = smem_u32(ring), b0 = smem_u32(tt);
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
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
                const uint32_t bhi = b0 + (ks >> 2) * (2 * kXTN * 128) + kin;
                umma_f16(dt, ad, smem_desc_sw128(bhi, 16, 1024), idesc, ks > 0 ? 1u : 0u);
                umma_f16(dt, ad, smem_desc_sw128(bhi + kXTN * 128, 16, 1024), idesc, 1u);
            }
            umma_commit(&empty[s]);
            umma_commit(&tfull[d]);
        }
    } else if (warp >= 2) {
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const int r = quad * 32 + lane;
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int v = find_volume(p.prefix, p.n_vol, g);
            const TcVol &vol = p.vols[v];
            const int64_t tile = g - __ldg(p.prefix + v);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&tfull[d], dph, 2)) break;
            tc_fence_after();
            const int64_t rows = vol.nz * vol.ny, nx = vol.nx;
            const int64_t row = (tile / vol.n_xt) * kTM + r;
            const int64_t xa = (tile % vol.n_xt) * kXTN + half * 64;
            uint32_t mw[2];
#pragma unroll
            for (int cc = 0; cc < 2; cc++) {
                const int64_t xb = xa + cc * 32;
                mw[cc] = (row < rows && xb < nx)
                             ? row_mask32<MAXI_MASK_BITPACKED>(vol.mask, row * nx + xb, nx - xb < 32 ? (int) (nx - xb) : 32,
                                                               rows * nx)
                             : 0u;
            }
            float ha[32], hb[32];
            __syncwarp();
            const uint32_t ta = tmem + ((uint32_t) (quad * 32) << 16) + d * kXTN + half * 64;
            tmem_ld32(ta, ha);
            tmem_ld32(ta + 32, hb);
            contig_epilogue64<S>(ha, hb, mw[0], mw[1], row, rows, nx, xa, p.inv_scale, p.error_feedback, p.final_pass,
                                 static_cast<uint16_t *>(vol.buf[p.in_buf ^ 1]), vol.out_u16, vol.field_out);
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

// ---- host --------------------------------------------------------------------------

static int strided_smem(int kp, int kpa) {
    return 1024 + 2 * kpa * kTM * 2 + kStages * (kTN / 64) * kp * 128 + 256 + kEpiWarps * kStageWarpBytes;
}
static int contig_smem(int kp, int kpa) { return 1024 + kpa * 2 * kXTN * 2 + kStages * (kpa / 64) * kTM * 128 + 256; }

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

// Fills the tile counts and the six tensor maps of one volume.
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
    vol.n_xc = (int) ceil_div(nx, kTN);
    vol.n_xt = (int) ceil_div(nx, kXTN);
    vol.cols_z = (int64_t) vol.n_xc * ny;
    vol.cols_y = (int64_t) vol.n_xc * nz;
    vol.tiles_x = (int64_t) vol.n_xt * ceil_div(nz * ny, kTM);
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
        if (enc(&vol.map[0][b], dt, 3, base, d3, s3, boxz, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.map[1][b], dt, 3, base, d3, s3, boxy, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
            enc(&vol.map[2][b], dt, 3, base, dx, sx, boxx, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return -1;
    }
    return 0;
}

cudaError_t tc_batch_pass(const TcVol *d_vols, const int64_t *d_prefix, int64_t total, int n_vol, int pass, int in_buf,
                          bool final_pass, const float *kernel, const TcGeometry &g, bool is_bf16, bool error_feedback,
                          cudaStream_t st) {
    if (total == 0) return cudaSuccess;
    BatchLaunch p{};
    p.vols = d_vols;
    p.prefix = d_prefix;
    p.n_vol = n_vol;
    p.pass = pass;
    p.in_buf = in_buf;
    p.final_pass = final_pass ? 1 : 0;
    p.radius = g.radius;
    p.ra = g.ra;
    p.kp = pass == 2 ? g.kp_contig : g.kp_strided;
    p.kpa = pass == 2 ? g.kpa_contig : g.kpa_strided;
    p.error_feedback = error_feedback ? 1 : 0;
    p.is_bf16 = is_bf16 ? 1 : 0;
    const float scale = is_bf16 ? 1.0f : 1024.0f;
    p.inv_scale = 1.0f / scale;
    tc_split_taps(kernel, g.radius, is_bf16, scale, p.hi, p.lo);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const unsigned grid = (unsigned) std::min<int64_t>(total, sms);
    cudaError_t e;
    if (pass == 2) {
        const int smem = contig_smem(p.kp, p.kpa);
        auto *k = is_bf16 ? tc_batch_contig<__nv_bfloat16> : tc_batch_contig<__half>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
        k<<<grid, kThreads, smem, st>>>(p);
    } else {
        const int smem = strided_smem(p.kp, p.kpa);
        auto *k = is_bf16 ? tc_batch_strided<__nv_bfloat16> : tc_batch_strided<__half>;
        if ((e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
        k<<<grid, kThreads, smem, st>>>(p);
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
