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
//      tensor memory, one lane per y-output, one accumulator per chunk.
//   2. Conversion warps read Y back lane by lane (tcgen05.ld), narrow it to the
//      16-bit storage type with error-feedback rounding along x (four chains of
//      8 per 32 columns, two voxels per instruction), zero the columns outside
//      the volume (the x pass's zero boundary), and write it packed two per
//      column (tcgen05.st) into its own tensor-memory region: the K-major
//      layout of an A operand in tensor memory.
//   3. x MMAs: D[o, x] = sum_j Y'[o, j] Tt[j, x] with the x Toeplitz Tt in
//      shared memory as the B operand (K-major), into the x accumulator.
//   4. Epilogue warps: re-illumination from the bit-packed mask, then either
//      the next field (error-feedback rounding, [y][z][x] or [z][y][x] rows) or,
//      on the last repetition, the uint16 output and the FP32 field.
//
// The field between the y and the x convolution is rounded to the storage
// type as the separate passes store it, so the arithmetic is that of the y
// pass followed by the x pass; only the HBM round trip of the intermediate
// field is gone (4 + 1/8 instead of 8 + 1/8 bytes per voxel for the two
// passes).  Coefficients: one 16-bit set rounded to keep the kernel's sum and
// second moment (tc_round_taps_matched).
//
// Tensor-core schedule.  Consecutive MMAs into one accumulator are bound by the
// MMA latency (about 130 cycles on B200 for N <= 192), so the MMA issuer keeps
// several accumulation chains in flight: the three 64-column y chunks of tile t
// (three accumulators) and the x MMAs of tile t - 1 (a fourth), one K step of
// each in turn.  That needs Y' of tile t - 1 to stay in place while tile t's y
// accumulates, hence its own region.  Tensor memory (512 columns): [0, 192) y
// accumulator, [192, 288) Y' packed, [288, 416) x accumulator, [416, 512) the
// y Toeplitz.  Warp roles: 0 TMA producer, 1 MMA issuer, 2-9 conversion (two
// per TMEM lane quadrant, 96 columns each), 10-17 epilogue (two per quadrant,
// 64 x-outputs each).  Every wait is bounded; on a timeout the kernel records a
// code in g_tc_error, lets the copies and MMAs it started finish (bounded) and
// winds down.
#pragma once

#include "tc_kernels.cuh"

namespace maxi {
namespace tc {

constexpr int kYxMaxStages = 8;                                  // F chunk ring (64 x-columns x KP rows each)
constexpr int kYxConvWarps = 8;                                  // two per TMEM lane quadrant
constexpr int kYxEpiWarps = 8;                                   // two per lane quadrant
constexpr int kYxThreads = 64 + 32 * (kYxConvWarps + kYxEpiWarps);  // 576
constexpr int kYxMaxChunks = 3;                                  // 64-column chunks of the x window (radius <= 32)
constexpr uint32_t kYxAccY = 0;                                  // y accumulators, up to 3 x 64 columns
constexpr uint32_t kYxYp = 192;                                  // Y' packed, up to 96 columns
constexpr uint32_t kYxAccX = 288;                                // x accumulator, 128 columns
constexpr uint32_t kYxToep = 416;                                // y Toeplitz, up to 96 columns
constexpr uint32_t kYxTmemCols = 512;

// Shared memory: x Toeplitz (kpa K x 128 rows), the F chunk ring of `stages`
// chunks, the barriers and the epilogue's store staging.
__host__ __device__ constexpr int yx_smem_bytes(int kp_y, int kpa_x, int stages) {
    return 1024 + kpa_x * kXTN * 2 + stages * kp_y * 128 + 1024 + kYxEpiWarps * kXStageWarpBytes;
}

// The deepest F ring (at most kYxMaxStages chunks) that fits `smem_max` bytes.
// A tile's y MMAs need its chunks together, so the ring holds two tiles'
// chunks where it can: the loads of the next tile run while this one multiplies.
__host__ __device__ constexpr int yx_stages(int kp_y, int kpa_x, int smem_max) {
    int st = kYxMaxStages;
    while (st > 3 && yx_smem_bytes(kp_y, kpa_x, st) > smem_max) st--;
    return st;
}

struct YxLaunch {
    PassTaps ty;  // y convolution: kp = 128 + 2R rounded to 16, kcols
    PassTaps tx;  // x convolution: ra, kp = 128 + RA + R rounded to 16, kpa
    int final_pass;
    int stages;         // F ring depth (chunks), at least the chunks of one tile
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

template <typename S, int FMT>
__global__ void __launch_bounds__(kYxThreads, 1)
tc_yx_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ YxLaunch p) {
    const PassTaps &ty = p.ty, &tx = p.tx;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *tt = smem;                                         // x Toeplitz, K-major, 128 rows
    uint8_t *ring = tt + tx.kpa * kXTN * 2;                     // a multiple of 16 KB: 1024-aligned
    const int chunk_bytes = ty.kp * 128;                        // 64 x-columns x KP rows of 16-bit
    const int nch = (tx.kp + 63) / 64;                          // chunks per tile (<= 3)
    const int ncc = (tx.kp + 31) / 32;                          // 32-column runs of Y' (<= 6)
    const int stages = p.stages;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + stages * chunk_bytes);
    uint64_t *full = bars, *empty = bars + kYxMaxStages;
    uint64_t *yfull = bars + 2 * kYxMaxStages;  // y accumulators complete (MMA commit)
    uint64_t *yfree = yfull + 1;                // y accumulators read (conversion warps)
    uint64_t *ypacked = yfull + 2;              // Y' written (conversion warps)
    uint64_t *ypfree = yfull + 3;               // Y' read by the x MMAs (MMA commit)
    uint64_t *xfull = yfull + 4;                // x accumulator complete (MMA commit)
    uint64_t *xempty = yfull + 5;               // x accumulator drained (epilogue warps)
    uint64_t *drain = yfull + 6;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(yfull + 7);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = p.n_tiles;
    const uint32_t n_tx = (uint32_t) p.n_tx, n_ty = (uint32_t) p.n_ty;

    for (int e = threadIdx.x; e < kXTN * tx.kpa; e += kYxThreads) {
        const int n = e / tx.kpa, j = e - n * tx.kpa;
        const int t = j - n - tx.ra + tx.radius;  // tap index 0..2R
        uint16_t v = 0;
        if (t >= 0 && t <= 2 * tx.radius && j < tx.kp) v = tx.hi[t];
        *reinterpret_cast<uint16_t *>(tt + sw128_kmajor_offset(n, j, kXTN)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(yfull, 1);
        mbar_init(yfree, kYxConvWarps);
        mbar_init(ypacked, kYxConvWarps);
        mbar_init(ypfree, 1);
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
    if (warp >= 2 && warp < 6) {
        // y Toeplitz into tensor memory (zero outside the band): one warp per quadrant.
        const int quad = warp & 3;
        const int o = quad * 32 + lane;
        for (int ch = 0; ch < ty.kcols / 32; ch++) {
            uint32_t r[32];
#pragma unroll
            for (int j = 0; j < 32; j++) {
                uint32_t v = 0;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int k = 2 * (ch * 32 + j) + e, t = k - o;
                    if (t >= 0 && t <= 2 * ty.radius && k < ty.kp) v |= (uint32_t) ty.hi[t] << (16 * e);
                }
                r[j] = v;
            }
            tmem_st32(tmem + ((uint32_t) (quad * 32) << 16) + kYxToep + ch * 32, r);
        }
        tmem_st_wait();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    // Tile g: plane z, y-tile, x-tile (x fastest, so the CTAs in flight work on
    // neighbouring tiles of one or two planes and share their halos in L2).
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
                const int s = (int) (cl % stages);
                const uint32_t ph = (uint32_t) ((cl / stages) & 1);
                if (!mbar_wait(&empty[s], ph ^ 1, 1)) { ok = false; break; }
                mbar_arrive_expect_tx(&full[s], chunk_bytes);
                tma_load_3d(ring + s * chunk_bytes, &tmap, x0 - tx.ra + 64 * c, y0 - ty.radius, z, &full[s]);
            }
        }
        // Let every copy this thread started land before the CTA can exit: the
        // last use of each ring stage (bounded, so an aborted run still ends).
        for (int64_t k = cl - stages; k < cl; k++)
            if (k >= 0) mbar_wait(&full[k % stages], (uint32_t) ((k / stages) & 1), 1);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.  Step tl issues the y MMAs of tile tl (one chain per chunk)
        // and the x MMAs of tile tl - 1, one K step of every chain in turn.
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc_y = idesc_f16(fmt, 0 /*A K-major*/, 1 /*B MN-major*/, kTM, 64);
        const uint32_t idesc_x = idesc_f16(fmt, 0 /*A K-major*/, 0 /*B K-major*/, kTM, kXTN);
        const uint32_t r0 = smem_u32(ring), t0 = smem_u32(tt);
        const int ksy = ty.kp / 16, ksx = tx.kp / 16, ks_max = ksy > ksx ? ksy : ksx;
        int64_t cl = 0;
        bool ok = true;
        for (int64_t tl = 0;; tl++) {
            const int64_t g = blockIdx.x + tl * (int64_t) gridDim.x;
            const bool has_y = g < total, has_x = tl > 0 && g - gridDim.x < total;
            if (!has_y && !has_x) break;
            int s[kYxMaxChunks] = {0, 0, 0};
            if (has_y) {
                for (int c = 0; c < nch && ok; c++) {
                    s[c] = (int) ((cl + c) % stages);
                    ok = mbar_wait(&full[s[c]], (uint32_t) (((cl + c) / stages) & 1), 1);
                }
                // the conversion warps have read the previous tile's y accumulators
                if (ok && tl > 0) ok = mbar_wait(yfree, (uint32_t) ((tl - 1) & 1), 3);
            }
            if (ok && has_x) {
                // Y' of tile tl - 1 is in place and the epilogue has drained the x accumulator
                ok = mbar_wait(ypacked, (uint32_t) ((tl - 1) & 1), 3) &&
                     mbar_wait(xempty, (uint32_t) (((tl - 1) & 1) ^ 1), 3);
            }
            if (!ok) break;
            tc_fence_after();
            for (int ks = 0; ks < ks_max; ks++) {
                if (has_y && ks < ksy) {
                    for (int c = 0; c < nch; c++) {
                        const uint64_t bd = smem_desc_sw128(r0 + s[c] * chunk_bytes, chunk_bytes, 1024);
                        umma_f16_ts(tmem + kYxAccY + 64 * c, tmem + kYxToep + ks * 8, bd + (uint64_t) (ks * 128),
                                    idesc_y, ks > 0 ? 1u : 0u);
                    }
                }
                if (has_x && ks < ksx) {
                    const uint32_t bhi = t0 + (ks >> 2) * (kXTN * 128) + (ks & 3) * 32;
                    umma_f16_ts(tmem + kYxAccX, tmem + kYxYp + ks * 8, smem_desc_sw128(bhi, 16, 1024), idesc_x,
                                ks > 0 ? 1u : 0u);
                }
            }
            if (has_y) {
                for (int c = 0; c < nch; c++) umma_commit(&empty[s[c]]);
                umma_commit(yfull);
                cl += nch;
            }
            if (has_x) {
                umma_commit(xfull);
                umma_commit(ypfree);
            }
        }
        // Every MMA this thread issued has completed before the CTA winds down.
        umma_commit(drain);
        mbar_wait(drain, 0, 2);
    } else if (warp >= 2 && warp < 2 + kYxConvWarps) {
        // Conversion: y accumulators (FP32) -> Y' (16-bit, packed).  The two warps
        // of a quadrant take the 32-column runs [3 half, 3 half + 3) of the window.
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lb = tmem + ((uint32_t) (quad * 32) << 16);
        const int c_lo = 3 * half, c_hi = ncc < c_lo + 3 ? ncc : c_lo + 3;
        int64_t tl = 0;
        bool ok = true;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x, tl++) {
            int z, y0, x0;
            decode(g, z, y0, x0);
            ok = __all_sync(0xffffffffu, mbar_wait(yfull, (uint32_t) (tl & 1), 2));
            if (!ok) break;
            tc_fence_after();
            for (int cc = c_lo; cc < c_hi || (cc == c_lo && c_lo >= c_hi); cc++) {
                const bool live = cc < c_hi;  // a half with no runs still signals
                float v[32];
                __syncwarp();
                if (live) tmem_ld32(lb + kYxAccY + 32 * cc, v);
                if (cc + 1 >= c_hi) {
                    // every read of this warp is done: the y accumulators may be reused
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(yfree);
                }
                if (cc == c_lo && tl > 0) {
                    // the x MMAs of the previous tile have read Y'
                    ok = __all_sync(0xffffffffu, mbar_wait(ypfree, (uint32_t) ((tl - 1) & 1), 2));
                    if (!ok) break;
                    tc_fence_after();
                }
                if (live) {
                    const int64_t xs = (int64_t) x0 - tx.ra + 32 * cc;
                    uint32_t d[16], w[16];
                    narrow32_quads<S, true>(v, ty.inv_scale, ty.error_feedback, 0u, live_bits(xs, p.nx), d);
                    quads_to_adjacent(d, w);
                    tmem_st16(lb + kYxYp + 16 * cc, w);
                }
            }
            if (!ok) break;
            tmem_st_wait();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(ypacked);
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
