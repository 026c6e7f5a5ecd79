// Fused y + x pass on the tensor cores for 16-bit field storage (radius <= 32).
//
// The separate y and x passes each read and write the whole field once; this
// kernel does both convolutions of one z-plane tile of 128 y-outputs x 128
// x-outputs without the intermediate field ever leaving the SM:
//
//   1. y MMAs: Y[o, j] = sum_k Ty[o, k] F[y0 - R + k, x0 - RA + j] for the 128
//      outputs o along y and KX = 128 + RA + R (rounded to 16) x-columns j --
//      the x pass's input window, halo included.  Ty (Toeplitz, in tensor
//      memory) is the A operand, F arrives by TMA in chunks of 64 x-columns x
//      KP = 128 + 2R rows (MN-major, 128-byte swizzle; rows and columns outside
//      the plane are zero-filled: the zero boundary).  Y accumulates in FP32 in
//      tensor memory, one lane per y-output.
//   2. Conversion warps read Y back lane by lane (tcgen05.ld), narrow it to the
//      16-bit storage type with error-feedback rounding along x (two chains per
//      32 columns, two voxels per instruction), zero the columns outside the
//      volume (the x pass's zero boundary), and write it back packed two per
//      column (tcgen05.st) over the first KX/2 columns of the accumulator: the
//      K-major layout of an A operand in tensor memory.
//   3. x MMAs: D[o, x] = sum_j Y'[o, j] Tt[j, x] with the x Toeplitz Tt in
//      shared memory as the B operand (K-major), into a second accumulator.
//   4. Epilogue warps: re-illumination from the bit-packed mask, then either
//      the next field (error-feedback rounding, [y][z][x] or [z][y][x] rows) or,
//      on the last repetition, the uint16 output and the FP32 field.
//
// The field between the y and the x convolution is rounded to the storage
// type exactly as the separate passes store it, so the arithmetic is that of
// the y pass followed by the x pass; only the HBM round trip of the
// intermediate field is gone (4 + 1/8 instead of 8 + 1/8 bytes per voxel for
// the two passes).  Coefficients are the high and low 16-bit halves of the
// kernel (two MMAs per K step) or, with hi_only, one 16-bit set whose
// rounding directions keep the kernel's sum and second moment (one MMA per
// K step: half the tensor-core work).
//
// Tensor memory (512 columns): [0, 192) y accumulator, then Y' packed over its
// first KX/2 columns; [192, 320) x accumulator; [320, 512) the y Toeplitz
// halves (96 columns each at radius 32).  Warp roles: 0 TMA producer, 1 MMA
// issuer, 2-9 conversion (two per TMEM lane quadrant, 32 columns of each
// 64-column chunk each), 10-17 epilogue (two per quadrant, 64 x-outputs each).
// The pipeline runs at chunk granularity: the y MMAs commit chunk by chunk,
// the conversion of a chunk starts while the next chunks multiply, and the x
// MMAs of a chunk start as soon as it is converted.  Every wait is bounded; on
// a timeout the kernel records a code in g_tc_error, lets the copies and MMAs
// it started finish (bounded) and winds down.
#pragma once

#include "tc_kernels.cuh"

namespace maxi {
namespace tc {

constexpr int kYxStages = 4;                                     // F chunk ring (64 x-columns x KP rows each)
constexpr int kYxConvWarps = 8;                                  // two per TMEM lane quadrant
constexpr int kYxEpiWarps = 8;                                   // two per lane quadrant
constexpr int kYxThreads = 64 + 32 * (kYxConvWarps + kYxEpiWarps);  // 576
constexpr int kYxMaxChunks = 3;                                  // 64-column chunks of the x window (radius <= 32)
constexpr uint32_t kYxAccY = 0;                                  // y accumulator, up to 192 columns
constexpr uint32_t kYxAccX = 192;                                // x accumulator, 128 columns
constexpr uint32_t kYxToep = 320;                                // y Toeplitz halves
constexpr uint32_t kYxTmemCols = 512;

// Shared memory: x Toeplitz (kpa K x 128 or 256 rows), the F chunk ring, the
// barriers and the epilogue's store staging.
__host__ __device__ constexpr int yx_smem_bytes(int kp_y, int kpa_x, bool hi_only) {
    return 1024 + kpa_x * (hi_only ? 1 : 2) * kXTN * 2 + kYxStages * kp_y * 128 + 1024 + kYxEpiWarps * kXStageWarpBytes;
}

struct YxLaunch {
    PassTaps ty;  // y convolution: kp = 128 + 2R rounded to 16, kcols
    PassTaps tx;  // x convolution: ra, kp = 128 + RA + R rounded to 16, kpa
    int hi_only;
    int final_pass;
    const void *mask;
    uint16_t *out;      // next field (not final): [z][y][x], or [y][z][x] rows when out_nz > 0
    uint16_t *out_u16;  // final
    float *field_out;   // final, optional
    int64_t nz, ny, nx, out_nz, out_z0;
    int n_ty, n_tx;
    int64_t n_tiles;
};

// Bits [lo, hi) of a 32-bit word (the voxels of a 32-voxel run inside [0, nx)).
__device__ __forceinline__ uint32_t live_bits(int64_t xs, int64_t nx) {
    if (xs >= 0 && xs + 32 <= nx) return 0xffffffffu;
    const int64_t lo = xs < 0 ? -xs : 0, hi = nx - xs < 32 ? nx - xs : 32;
    if (hi <= lo) return 0u;
    const uint32_t upto = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
    return upto & ~((1u << lo) - 1u);
}

// Named barrier of the two conversion warps of one TMEM lane quadrant that
// also ANDs `v` over both: the pair leaves a wait that timed out together.
__device__ __forceinline__ bool pair_barrier_and(int quad, bool v) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred p, q;\n setp.ne.u32 p, %2, 0;\n bar.red.and.pred q, %1, 64, p;\n selp.u32 %0, 1, 0, q;\n}\n"
        : "=r"(r) : "r"(1 + quad), "r"((uint32_t) v) : "memory");
    return r != 0;
}

template <typename S, int FMT>
__global__ void __launch_bounds__(kYxThreads, 1)
tc_yx_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ YxLaunch p) {
    const PassTaps &ty = p.ty, &tx = p.tx;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    const int tt_rows = p.hi_only ? kXTN : 2 * kXTN;          // x Toeplitz rows: hi (and lo)
    uint8_t *tt = smem;
    uint8_t *ring = tt + tx.kpa * tt_rows * 2;                 // a multiple of 16 KB: 1024-aligned
    const int chunk_bytes = ty.kp * 128;                        // 64 x-columns x KP rows of 16-bit
    const int nch = (tx.kp + 63) / 64;                          // chunks per tile (<= 3)
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kYxStages * chunk_bytes);
    uint64_t *full = bars, *empty = bars + kYxStages;
    uint64_t *ychunk = bars + 2 * kYxStages;                    // [kYxMaxChunks]: y chunk accumulated
    uint64_t *ypacked = ychunk + kYxMaxChunks;                  // [kYxMaxChunks]: chunk converted to Y'
    uint64_t *xfull = ypacked + kYxMaxChunks, *xempty = xfull + 1, *drain = xfull + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(xfull + 3);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = p.n_tiles;
    const uint32_t n_tx = (uint32_t) p.n_tx, n_ty = (uint32_t) p.n_ty;

    for (int e = threadIdx.x; e < tt_rows * tx.kpa; e += kYxThreads) {
        const int n = e / tx.kpa, j = e - n * tx.kpa;
        const int o = n & (kXTN - 1);
        const int t = j - o - tx.ra + tx.radius;  // tap index 0..2R
        uint16_t v = 0;
        if (t >= 0 && t <= 2 * tx.radius && j < tx.kp) v = n < kXTN ? tx.hi[t] : tx.lo[t];
        *reinterpret_cast<uint16_t *>(tt + sw128_kmajor_offset(n, j, tt_rows)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kYxStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int c = 0; c < kYxMaxChunks; c++) { mbar_init(&ychunk[c], 1); mbar_init(&ypacked[c], kYxConvWarps); }
        mbar_init(xfull, 1);
        mbar_init(xempty, kYxEpiWarps);
        mbar_init(drain, 1);
        fence_barrier_init();
        prefetch_tmap(&tmap);
    }
    __syncwarp();
    if (warp == 0) {
        tmem_alloc(tmem_slot, kYxTmemCols);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp >= 2 && warp < 10) {
        // y Toeplitz halves into tensor memory (zero outside the band): the two
        // warps of a lane quadrant write Ty_hi and Ty_lo of its 32 rows.
        const int quad = warp & 3, lo_half = (warp - 2) >> 2;
        if (!(lo_half && p.hi_only)) {
            const int o = quad * 32 + lane;
            const uint16_t *taps = lo_half ? ty.lo : ty.hi;
            for (int ch = 0; ch < ty.kcols / 32; ch++) {
                uint32_t r[32];
#pragma unroll
                for (int j = 0; j < 32; j++) {
                    uint32_t v = 0;
#pragma unroll
                    for (int e = 0; e < 2; e++) {
                        const int k = 2 * (ch * 32 + j) + e, t = k - o;
                        if (t >= 0 && t <= 2 * ty.radius && k < ty.kp) v |= (uint32_t) taps[t] << (16 * e);
                    }
                    r[j] = v;
                }
                tmem_st32(tmem + ((uint32_t) (quad * 32) << 16) + kYxToep + (lo_half ? ty.kcols : 0) + ch * 32, r);
            }
            tmem_st_wait();
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    // Tile g: plane z, y-tile ty_, x-tile tx_ (x fastest, so the CTAs in flight
    // work on neighbouring tiles of one or two planes and share their halos in L2).
    auto decode = [&](int64_t g, int &z, int &y0, int &x0) {
        const uint32_t gg = (uint32_t) g, rest = gg / n_tx, t_y = rest % n_ty;
        x0 = (int) (gg - rest * n_tx) * kXTN;
        y0 = (int) t_y * kTM;
        z = (int) (rest / n_ty);
    };

    if (warp == 0 && lane == 0) {
        // TMA producer: nch chunks per tile into the ring; L2 prefetch ahead.
        int64_t cl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x) {
            int z, y0, x0;
            const int64_t gp = g + kPrefetch * (int64_t) gridDim.x;
            if (gp < total) {
                decode(gp, z, y0, x0);
                for (int c = 0; c < nch; c++) tma_prefetch_3d(&tmap, x0 - tx.ra + 64 * c, y0 - ty.radius, z);
            }
            decode(g, z, y0, x0);
            for (int c = 0; c < nch; c++, cl++) {
                const int s = (int) (cl % kYxStages);
                const uint32_t ph = (uint32_t) ((cl / kYxStages) & 1);
                if (!mbar_wait(&empty[s], ph ^ 1, 1)) { ok = false; break; }
                mbar_arrive_expect_tx(&full[s], chunk_bytes);
                tma_load_3d(ring + s * chunk_bytes, &tmap, x0 - tx.ra + 64 * c, y0 - ty.radius, z, &full[s]);
            }
        }
        // Let every copy this thread started land before the CTA can exit: the
        // last use of each ring stage (bounded, so an aborted run still ends).
        for (int64_t k = cl - kYxStages; k < cl; k++)
            if (k >= 0) mbar_wait(&full[k % kYxStages], (uint32_t) ((k / kYxStages) & 1), 1);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.  Per tile: the y MMAs chunk by chunk (each chunk committed
        // on its own barrier, so its conversion starts while the next chunks
        // multiply), then the x MMAs chunk by chunk as each chunk of Y' lands.
        // The y MMAs of a tile overwrite the previous tile's Y', which the x MMAs
        // issued before them have read (tcgen05.mma of one thread run in issue order).
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc_y = idesc_f16(fmt, 0 /*A K-major*/, 1 /*B MN-major*/, kTM, 64);
        const uint32_t idesc_x = idesc_f16(fmt, 0 /*A K-major*/, 0 /*B K-major*/, kTM, kXTN);
        const uint32_t r0 = smem_u32(ring), t0 = smem_u32(tt);
        const uint32_t a_hi = tmem + kYxToep, a_lo = a_hi + ty.kcols;
        const int ksx = tx.kp / 16;
        int64_t cl = 0, tl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x, tl++) {
            const uint32_t ph = (uint32_t) (tl & 1);
            for (int c = 0; c < nch; c++, cl++) {
                const int s = (int) (cl % kYxStages);
                if (!mbar_wait(&full[s], (uint32_t) ((cl / kYxStages) & 1), 1)) { ok = false; break; }
                tc_fence_after();
                const uint64_t bd = smem_desc_sw128(r0 + s * chunk_bytes, chunk_bytes, 1024);
                const uint32_t d = tmem + kYxAccY + 64 * c;
                for (int ks = 0; ks < ty.kp / 16; ks++) {
                    umma_f16_ts(d, a_hi + ks * 8, bd + (uint64_t) (ks * 128), idesc_y, ks > 0 ? 1u : 0u);
                    if (!p.hi_only) umma_f16_ts(d, a_lo + ks * 8, bd + (uint64_t) (ks * 128), idesc_y, 1u);
                }
                umma_commit(&empty[s]);
                umma_commit(&ychunk[c]);
            }
            if (!ok) break;
            if (!mbar_wait(xempty, ph ^ 1, 3)) break;  // the epilogue has drained the x accumulator
            const uint32_t dx = tmem + kYxAccX;
            for (int c = 0; c < nch && ok; c++) {
                if (!mbar_wait(&ypacked[c], ph, 3)) { ok = false; break; }
                tc_fence_after();
                for (int ks = 4 * c; ks < 4 * c + 4 && ks < ksx; ks++) {
                    const uint32_t kin = (ks & 3) * 32;
                    const uint32_t bhi = t0 + (ks >> 2) * (tt_rows * 128) + kin;
                    umma_f16_ts(dx, tmem + kYxAccY + ks * 8, smem_desc_sw128(bhi, 16, 1024), idesc_x, ks > 0 ? 1u : 0u);
                    if (!p.hi_only)
                        umma_f16_ts(dx, tmem + kYxAccY + ks * 8, smem_desc_sw128(bhi + kXTN * 128, 16, 1024), idesc_x, 1u);
                }
            }
            if (!ok) break;
            umma_commit(xfull);
        }
        // Every MMA this thread issued has completed before the CTA winds down.
        umma_commit(drain);
        mbar_wait(drain, 0, 2);
    } else if (warp >= 2 && warp < 2 + kYxConvWarps) {
        // Conversion: y accumulator (FP32) -> Y' (16-bit, packed) in place, one
        // 64-column chunk at a time; the two warps of a quadrant take 32 columns
        // each.  Chunk c's packed words land on FP32 columns of chunk c / 2: both
        // warps have read those (the pair barrier orders the reads of chunk c
        // before either warp's writes of chunk c).
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lb = tmem + ((uint32_t) (quad * 32) << 16);
        int64_t tl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x, tl++) {
            int z, y0, x0;
            decode(g, z, y0, x0);
            for (int c = 0; c < nch; c++) {
                // warp-uniform, then pair-uniform outcome of the wait: both warps
                // of the pair reach the barrier either way and leave together
                ok = __all_sync(0xffffffffu, mbar_wait(&ychunk[c], (uint32_t) (tl & 1), 2));
                tc_fence_after();
                float v[32];
                __syncwarp();
                if (ok) tmem_ld32(lb + kYxAccY + 64 * c + 32 * half, v);
                ok = pair_barrier_and(quad, ok);
                if (!ok) break;
                const int64_t xs = (int64_t) x0 - tx.ra + 64 * c + 32 * half;
                uint32_t d[16], w[16];
                narrow32_pairs<S, true>(v, ty.inv_scale, ty.error_feedback, 0u, live_bits(xs, p.nx), d);
                pairs_to_adjacent(d, w);
                tmem_st16(lb + kYxAccY + 32 * c + 16 * half, w);
                tmem_st_wait();
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&ypacked[c]);
            }
        }
    } else if (warp >= 2 + kYxConvWarps) {
        // Epilogue: x accumulator -> re-illumination -> next field / final outputs.
        const int ew = warp - 2 - kYxConvWarps;
        const int quad = warp & 3, part = ew >> 2;  // part: x-outputs part * 64 .. + 64 of the tile
        const uint32_t lb = tmem + ((uint32_t) (quad * 32) << 16);
        uint8_t *stg = stage_out + ew * kXStageWarpBytes;
        const int64_t n_vox = p.nz * p.ny * p.nx, rows = p.nz * p.ny;
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            int z, y0, x0;
            decode(g, z, y0, x0);
            const int64_t y = y0 + quad * 32 + lane;
            const bool live_row = y < p.ny;
            const int64_t row = (int64_t) z * p.ny + y;
            MaskWords mw[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int64_t xb = x0 + part * 64 + 32 * k;
                if (live_row && xb < p.nx)
                    mw[k] = load_mask_words<FMT>(p.mask, row * p.nx + xb, p.nx - xb < 32 ? (int) (p.nx - xb) : 32, n_vox);
            }
            if (!__all_sync(0xffffffffu, mbar_wait(xfull, (uint32_t) (tl & 1), 2))) break;
            tc_fence_after();
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int64_t xb = x0 + part * 64 + 32 * k;
                float h[32];
                __syncwarp();
                tmem_ld32(lb + kYxAccX + part * 64 + 32 * k, h);
                const uint32_t m = mask_flags<FMT>(mw[k], p.mask);
                if (p.final_pass) {
                    contig_final32(h, m, live_row ? row : rows, rows, p.nx, xb, tx.inv_scale, p.out_u16, p.field_out);
                } else if (xb < p.nx) {  // warp-uniform
                    uint32_t d[16], q[16];
                    narrow32_pairs<S, true>(h, tx.inv_scale, tx.error_feedback, m, 0xffffffffu, d);
                    pairs_to_adjacent(d, q);
                    const int64_t oi = !live_row ? -1
                                       : p.out_nz == 0 ? row * p.nx + xb
                                                        : ((y * p.out_nz + p.out_z0 + z) * p.nx) + xb;
                    __syncwarp();
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        *reinterpret_cast<uint4 *>(stg + lane * 64 + ((i ^ ((lane >> 1) & 3)) << 4)) =
                            make_uint4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
                    __syncwarp();
                    const int sub = lane & 3, rsub = lane >> 2;
#pragma unroll
                    for (int r4 = 0; r4 < 4; r4++) {
                        const int rr = r4 * 8 + rsub;
                        const int64_t o = __shfl_sync(0xffffffffu, oi, rr);
                        const uint4 wv = *reinterpret_cast<const uint4 *>(stg + rr * 64 + ((sub ^ ((rr >> 1) & 3)) << 4));
                        if (o >= 0 && xb + sub * 8 < p.nx) *reinterpret_cast<uint4 *>(p.out + o + sub * 8) = wv;
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(xempty);
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kYxTmemCols);
    }
}

}  // namespace tc
}  // namespace maxi
