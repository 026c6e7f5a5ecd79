// Fused y + x pass on the tensor cores for 16-bit field storage (radius <= 32).
//
// The separate y and x passes each read and write the whole field once; this
// kernel does both convolutions of one z-plane tile of 128 y-outputs x 128
// x-outputs without the intermediate field ever leaving the SM:
//
//   1. y MMA: Y[o, j] = sum_k T[o, k] F[y0 - RA + k, x0 - RA + j] for the 128
//      outputs o along y and the KP = 128 + RA + R (rounded to 16) x-columns j
//      of the x pass's input window, halo included (RA = R rounded up to 8, the
//      16-byte alignment of the window's first x).  T[o, k] = tap[k - o - RA + R]
//      (zero outside the band) is the A operand in shared memory; F arrives by
//      TMA as KP rows x KP columns (64-column boxes, MN-major, 128-byte swizzle;
//      rows and columns outside the plane are zero-filled: the zero boundary).
//      One accumulation chain of N = KP columns, FP32, in tensor memory.
//   2. Conversion warps read Y back (tcgen05.ld), narrow it to the 16-bit
//      storage type with error-feedback rounding along x (chains of 8 voxels,
//      two voxels per instruction) and write it packed two per column
//      (tcgen05.st) into one of two Y' buffers: the K-major layout of an A
//      operand in tensor memory.  Columns outside the volume hold exact zeros
//      (their F columns are zero and nx is a multiple of 8, so every chain lies
//      wholly inside or wholly outside): the x pass's zero boundary.
//   3. x MMA: D[o, x] = sum_j Y'[o, j] T[x, j], the same Toeplitz matrix in
//      shared memory as the B operand (K-major), into the x accumulator.
//   4. Epilogue warps: re-illumination from the bit-packed mask, then either
//      the next field (error-feedback rounding, [y][z][x] or [z][y][x] rows) or,
//      on the last repetition, the uint16 output and the FP32 field.
//
// The field between the y and the x convolution is rounded to the storage
// type as the separate passes store it, so the arithmetic is that of the y
// pass followed by the x pass; only the HBM round trip of the intermediate
// field is gone (4 + 1/8 instead of 8 + 1/8 bytes per voxel for the two
// passes).  Coefficients: one 16-bit set rounded, at a searched scale, to keep
// the kernel's sum and second moment (tc_round_taps_scaled).
//
// Tensor-core schedule.  Narrow MMAs are bound by their issue (one thread
// issues an M = 128, N = 64 MMA about every 60 cycles, twice the tensor pipe's
// time), wide ones by the pipe: so every product is one chain of the widest N
// (KP / 16 MMAs each for y and x per tile), and the y and the x MMAs have an
// issuing thread each, so that neither waits on the other's issue.  The
// conversion of tile t runs while the tensor cores do x(t - 1) and writes the
// other Y' buffer.  Tensor memory (512 columns): [0, 192) y accumulator,
// [192, 384) the two Y' buffers, [384, 512) x accumulator.  Warp roles: 0 TMA
// producer, 1 y MMA issuer, 2-9 conversion (two per TMEM lane quadrant), 10-17
// epilogue (two per quadrant, 64 x-outputs each), 18 x MMA issuer.  Every wait
// is bounded; on a timeout the kernel records a code in g_tc_error, lets the
// copies and MMAs it started finish (bounded) and winds down.
#pragma once

#include "tc_kernels.cuh"

namespace maxi {
namespace tc {

constexpr int kYxMaxStages = 4;                                  // F tile ring
constexpr int kYxConvWarps = 8;                                  // two per TMEM lane quadrant
constexpr int kYxEpiWarps = 8;                                   // two per lane quadrant
constexpr int kYxXWarp = 2 + kYxConvWarps + kYxEpiWarps;       // x MMA issuer (warp 18)
constexpr int kYxThreads = 32 * (kYxXWarp + 1);                  // 608
constexpr int kYxMaxCols = 192;                                  // KP for radius <= 32
constexpr uint32_t kYxAccY = 0;                                  // y accumulator, KP columns
constexpr uint32_t kYxYp = 192;                                  // two Y' buffers of KP / 2 columns
constexpr uint32_t kYxYpCols = 96;
constexpr uint32_t kYxAccX = 384;                                // x accumulator, 128 columns
constexpr uint32_t kYxTmemCols = 512;

// Output order of the Toeplitz rows: row n of the matrix in shared memory is
// output (n & ~31) + P(n & 31) with P(2j) = j and P(2j + 1) = 16 + j.  The y
// MMAs then leave y-output P(l) in TMEM lane l of each quadrant, and the x MMAs
// leave x-output P(c) in column c of each 32-column run, so that the voxels the
// epilogue rounds together (j and 16 + j of a run: two error-feedback chains)
// arrive in adjacent registers of its tensor-memory loads.
__host__ __device__ constexpr int yx_out_perm(int n) { return (n & ~31) | (((n & 31) >> 1) + ((n & 1) << 4)); }

// One F tile: ceil(KP / 64) boxes of 64 x-columns x KP rows.
__host__ __device__ constexpr int yx_tile_bytes(int kp) { return ((kp + 63) / 64) * kp * 128; }

// Shared memory: the Toeplitz matrix (kpa K x 128 rows), the F tile ring of
// `stages` tiles, the barriers and the epilogue's store staging (two 32 x 32
// chunks per warp, the sources of its TMA stores).
__host__ __device__ constexpr int yx_smem_bytes(int kp, int kpa, int stages) {
    return 1024 + kpa * kXTN * 2 + stages * yx_tile_bytes(kp) + 1024 + kYxEpiWarps * 2 * kXStageWarpBytes;
}

// The deepest F ring (2 .. kYxMaxStages tiles) that fits `smem_max` bytes.
__host__ __device__ constexpr int yx_stages(int kp, int kpa, int smem_max) {
    int st = kYxMaxStages;
    while (st > 2 && yx_smem_bytes(kp, kpa, st) > smem_max) st--;
    return st;
}

// One tile of the fused kernel: where its volume's field, mask and outputs
// are, and which plane, y-tile and x-tile it is.
struct YxTile {
    const CUtensorMap *in;   // input field (x, y, z), box 64 x KP x 1
    const CUtensorMap *out;  // next field's store map, box 32 x 32: (x, y, z), or (x, z, y) when rows_yzx
    const void *mask;
    uint16_t *out_u16;       // final
    float *field_out;        // final, optional
    int64_t ny, nx, rows, n_vox;
    int z, y0, x0, rows_yzx;
};

// Tile g of a volume: x-tile g % n_tx, then y-tile, then plane (x fastest, so
// the CTAs in flight work on neighbouring tiles of one or two planes and share
// their halos in L2).  The divisions use the multiply below: floor(g / d) for
// g < 2^32 as the high word of g * M, M = ceil(2^64 / d)
// (d >= 2; yx_div_magic(1) = 0 marks d = 1): the product's excess over g / d
// stays below g / 2^64 < 1 / d, so the floor is exact.
__host__ __device__ constexpr uint64_t yx_div_magic(uint32_t d) {
    return d <= 1 ? 0ull : ~0ull / d + 1ull;
}
__device__ __forceinline__ uint32_t yx_div(uint32_t g, uint32_t d, uint64_t magic) {
    return magic ? (uint32_t) __umul64hi((uint64_t) g, magic) : g;
}

// One volume: maps are kernel parameters.  The next field goes to [z][y][x]
// rows, or to [y][z][x] rows (rows_yzx; the store map covers the plane window).
struct OneVolumeYx {
    struct Cursor {};
    const void *mask;
    uint16_t *out_u16;
    float *field_out;
    int64_t nz, ny, nx;
    int n_ty, n_tx, rows_yzx;
    int64_t n_tiles;
    uint64_t magic_tx, magic_ty;  // yx_div_magic(n_tx), yx_div_magic(n_ty)
    __device__ __forceinline__ int64_t total() const { return n_tiles; }
    __device__ __forceinline__ YxTile tile(int64_t g, const CUtensorMap *in, const CUtensorMap *out, Cursor &) const {
        YxTile t;
        t.in = in;
        t.out = out;
        t.mask = mask;
        t.out_u16 = out_u16;
        t.field_out = field_out;
        t.ny = ny;
        t.nx = nx;
        t.rows = nz * ny;
        t.n_vox = nz * ny * nx;
        t.rows_yzx = rows_yzx;
        const uint32_t gg = (uint32_t) g;
        const uint32_t rest = yx_div(gg, (uint32_t) n_tx, magic_tx);
        const uint32_t z = yx_div(rest, (uint32_t) n_ty, magic_ty);
        t.x0 = (int) (gg - rest * (uint32_t) n_tx) * kXTN;
        t.y0 = (int) (rest - z * (uint32_t) n_ty) * kTM;
        t.z = (int) z;
        return t;
    }
};

// Many volumes (a batch group): maps and sizes from the device table; tile g
// lies in the volume whose prefix-sum range holds it.  The next field goes to
// the volume's other buffer in [y][z][x] rows.
struct ManyVolumesYx {
    const TcVol *vols;
    const int64_t *prefix;  // n_vol + 1 prefix sums of the volumes' tiles
    int n_vol, in_buf;
    struct Cursor {
        int64_t lo = 0, hi = 0;  // the current volume's tiles [lo, hi)
        int v = 0;
    };
    __device__ __forceinline__ int64_t total() const { return __ldg(prefix + n_vol); }
    __device__ __forceinline__ YxTile tile(int64_t g, const CUtensorMap *, const CUtensorMap *, Cursor &cur) const {
        if (g < cur.lo || g >= cur.hi) {
            cur.v = find_volume(prefix, n_vol, g);
            cur.lo = __ldg(prefix + cur.v);
            cur.hi = __ldg(prefix + cur.v + 1);
        }
        const TcVol &vol = vols[cur.v];
        YxTile t;
        t.in = &vol.map[1][in_buf];
        t.out = &vol.yxrows[in_buf ^ 1];
        t.mask = vol.mask;
        t.out_u16 = vol.out_u16;
        t.field_out = vol.field_out;
        t.ny = vol.ny;
        t.nx = vol.nx;
        t.rows = vol.nz * vol.ny;
        t.n_vox = vol.nz * vol.ny * vol.nx;
        t.rows_yzx = 1;
        const uint32_t gg = (uint32_t) (g - cur.lo);
        const uint32_t rest = yx_div(gg, (uint32_t) vol.n_xt, vol.magic_xt);
        const uint32_t z = yx_div(rest, (uint32_t) vol.n_at_y, vol.magic_at_y);
        t.x0 = (int) (gg - rest * (uint32_t) vol.n_xt) * kXTN;
        t.y0 = (int) (rest - z * (uint32_t) vol.n_at_y) * kTM;
        t.z = (int) z;
        return t;
    }
};

template <class Sched>
struct YxLaunch {
    PassTaps t;  // ra = RA, kp = KP = 128 + RA + R rounded to 16, one coefficient set
    int final_pass;     // selects the FINAL instantiation
    int stages;         // F ring depth (tiles)
    Sched sched;
};

// FINAL: the last repetition (uint16 output and FP32 field instead of the next
// 16-bit field); a template parameter so that each form holds only its own
// epilogue's registers.
template <typename S, int FMT, bool FINAL, class Sched>
__global__ void __launch_bounds__(kYxThreads, 1)
tc_yx_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap omap,
             const __grid_constant__ YxLaunch<Sched> p) {
    const PassTaps &tp = p.t;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *tt = smem;                                         // Toeplitz, K-major, 128 rows
    uint8_t *ring = tt + tp.kpa * kXTN * 2;                     // a multiple of 16 KB: 1024-aligned
    const int kp = tp.kp;
    const int chunk_bytes = kp * 128;                           // 64 x-columns x KP rows of 16-bit
    const int nch = (kp + 63) / 64;                             // boxes per tile (<= 3)
    const int tile_bytes = nch * chunk_bytes;
    const int ncc = (kp + 31) / 32;                             // 32-column runs of Y (5 or 6)
    const int stages = p.stages;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + stages * tile_bytes);
    uint64_t *full = bars, *empty = bars + kYxMaxStages;
    uint64_t *yfull = bars + 2 * kYxMaxStages;  // y accumulator complete (MMA commit)
    uint64_t *yfree = yfull + 1;                // y accumulator read (conversion warps)
    uint64_t *ypacked = yfull + 2;              // [2] Y' buffer written (conversion warps)
    uint64_t *xfull = yfull + 4;                // x accumulator complete (x MMA commit)
    uint64_t *xempty = yfull + 5;               // x accumulator read (epilogue warps)
    uint64_t *ypfree = yfull + 6;               // [2] Y' buffer read by the x MMAs (x MMA commit)
    uint64_t *drain = yfull + 8;                // [2] every MMA of the y / x issuer complete
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(yfull + 10);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Sched &sched = p.sched;
    const int64_t total = sched.total();

    // T[n, j] = tap[j - n - RA + R]: the y pass's A (row n = output o, K = j)
    // and the x pass's B (row n = x-output, K = j) alike.
    for (int e = threadIdx.x; e < kXTN * tp.kpa; e += kYxThreads) {
        const int n = e / tp.kpa, j = e - n * tp.kpa;
        const int t = j - yx_out_perm(n) - tp.ra + tp.radius;  // tap index 0..2R
        uint16_t v = 0;
        if (t >= 0 && t <= 2 * tp.radius && j < kp) v = tp.hi[t];
        *reinterpret_cast<uint16_t *>(tt + sw128_kmajor_offset(n, j, kXTN)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < stages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(yfull, 1);
        mbar_init(yfree, kYxConvWarps);
        mbar_init(&ypacked[0], kYxConvWarps);
        mbar_init(&ypacked[1], kYxConvWarps);
        mbar_init(xfull, 1);
        mbar_init(xempty, kYxEpiWarps);
        mbar_init(&ypfree[0], 1);
        mbar_init(&ypfree[1], 1);
        mbar_init(&drain[0], 1);
        mbar_init(&drain[1], 1);
        fence_barrier_init();
        if (std::is_same<Sched, OneVolumeYx>::value) {
            prefetch_tmap(&tmap);
            if (!FINAL) prefetch_tmap(&omap);
        }
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

    if (warp == 0 && lane == 0) {
        // TMA producer: one F tile (nch boxes) per ring stage; L2 prefetch ahead.
        // The stage and its phase advance incrementally (the ring depth is a
        // run-time value: no 64-bit division per tile).
        int64_t tl = 0;
        int s = 0;
        uint32_t ph = 0;
        typename Sched::Cursor cur, pcur;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int64_t gp = g + kPrefetch * (int64_t) gridDim.x;
            if (gp < total) {
                const YxTile q = sched.tile(gp, &tmap, &omap, pcur);
                for (int c = 0; c < nch; c++) tma_prefetch_3d(q.in, q.x0 - tp.ra + 64 * c, q.y0 - tp.ra, q.z);
            }
            const YxTile t = sched.tile(g, &tmap, &omap, cur);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) break;
            mbar_arrive_expect_tx(&full[s], tile_bytes);
            for (int c = 0; c < nch; c++)
                tma_load_3d(ring + s * tile_bytes + c * chunk_bytes, t.in, t.x0 - tp.ra + 64 * c, t.y0 - tp.ra, t.z,
                            &full[s]);
            if (++s == stages) s = 0, ph ^= 1;
        }
        // Let every copy this thread started land before the CTA can exit: the
        // last use of each ring stage (bounded, so an aborted run still ends).
        for (int64_t k = tl - stages; k < tl; k++)
            if (k >= 0) mbar_wait(&full[k % stages], (uint32_t) ((k / stages) & 1), 1);
    } else if ((warp == 1 || warp == kYxXWarp) && lane == 0) {
        // MMA issuers: the y MMAs (warp 1) and the x MMAs (warp 18) have an
        // issuing thread each; their ordering is through the barriers.
        const bool is_y = warp == 1;
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc_y = idesc_f16(fmt, 0 /*A K-major*/, 1 /*B MN-major*/, kTM, (uint32_t) kp);
        const uint32_t idesc_x = idesc_f16(fmt, 0 /*A K-major*/, 0 /*B K-major*/, kTM, kXTN);
        // T: K step ks at 64-element block ks / 4 (16 KB each), 32 bytes per 16 K inside it.
        const uint64_t t_desc = smem_desc_sw128(smem_u32(tt), 16, 1024);
        const uint32_t r0 = smem_u32(ring);
        const int ks_n = kp / 16;
        int s = 0;  // ring stage of tile tl and its phase, advanced incrementally
        uint32_t ph = 0;
        for (int64_t tl = 0; blockIdx.x + tl * (int64_t) gridDim.x < total; tl++) {
            if (is_y) {
                // y(tl): its F tile has landed and the conversion warps have read y(tl - 1)
                bool ok = mbar_wait(&full[s], ph, 1);
                if (ok && tl > 0) ok = mbar_wait(yfree, (uint32_t) ((tl - 1) & 1), 3);
                if (!ok) break;
                tc_fence_after();
                // F: MN-major, 64-column atoms chunk_bytes apart (LBO), 8-row groups 1 KB apart (SBO).
                const uint64_t f_desc = smem_desc_sw128(r0 + s * tile_bytes, chunk_bytes, 1024);
                for (int ks = 0; ks < ks_n; ks++)
                    umma_f16(tmem + kYxAccY, t_desc + (uint64_t) ((ks >> 2) * 1024 + (ks & 3) * 2),
                             f_desc + (uint64_t) (ks * 128), idesc_y, ks > 0 ? 1u : 0u);
                umma_commit(&empty[s]);
                umma_commit(yfull);
                if (++s == stages) s = 0, ph ^= 1;
            } else {
                // x(tl): Y' of tile tl is in place (one barrier per buffer: the
                // conversion warps cannot complete a second phase of it before this
                // wait, since that needs x(tl) itself) and the epilogue has read
                // x(tl - 1)
                const int b = (int) (tl & 1);
                if (!(mbar_wait(&ypacked[b], (uint32_t) ((tl >> 1) & 1), 3) &&
                      mbar_wait(xempty, (uint32_t) ((tl & 1) ^ 1), 3)))
                    break;
                tc_fence_after();
                const uint32_t yp = tmem + kYxYp + (uint32_t) b * kYxYpCols;
                for (int ks = 0; ks < ks_n; ks++)
                    umma_f16_ts(tmem + kYxAccX, yp + ks * 8, t_desc + (uint64_t) ((ks >> 2) * 1024 + (ks & 3) * 2),
                                idesc_x, ks > 0 ? 1u : 0u);
                umma_commit(xfull);
                umma_commit(&ypfree[b]);
            }
        }
        // Every MMA this thread issued has completed before the CTA winds down.
        umma_commit(&drain[is_y ? 0 : 1]);
        mbar_wait(&drain[is_y ? 0 : 1], 0, 2);
    } else if (warp >= 2 && warp < 2 + kYxConvWarps) {
        // Conversion: y accumulator (FP32) -> Y' (16-bit, packed).  The two warps
        // of a quadrant take the 32-column runs [3 half, 3 half + 3) of the
        // window (two or three of them): a third run first, then two together,
        // whose reads free the y accumulator for y(tl + 1).  Y' of tile tl goes
        // to buffer tl & 1, once x(tl - 2) has read it.
        const int quad = warp & 3, half = (warp - 2) >> 2;
        const uint32_t lb = tmem + ((uint32_t) (quad * 32) << 16);
        const int c0 = 3 * half, c1 = ncc < c0 + 3 ? ncc : c0 + 3;  // 2 or 3 runs
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            if (!__all_sync(0xffffffffu, mbar_wait(yfull, (uint32_t) (tl & 1), 2))) break;
            tc_fence_after();
            const uint32_t yp = lb + kYxYp + (uint32_t) (tl & 1) * kYxYpCols;
            // Before the first write to the Y' buffer: x(tl - 2), its last reader, has completed.
            bool yp_free = tl < 2, ok = true;
            auto wait_yp = [&]() {
                if (yp_free) return;
                ok = __all_sync(0xffffffffu, mbar_wait(&ypfree[tl & 1], (uint32_t) (((tl >> 1) - 1) & 1), 2));
                tc_fence_after();
                yp_free = true;
            };
            // A third run first, narrowed and held as pairs, so that the last two
            // reads come together and free the y accumulator for y(tl + 1) before
            // this warp waits for its Y' buffer.
            const bool third = c1 == c0 + 3;
            uint32_t w3[16];
            if (third) {
                float v[32];
                __syncwarp();
                tmem_ld32(lb + kYxAccY + 32 * (c0 + 2), v);
                uint32_t d[16];
                narrow32_quads<S>(v, tp.inv_scale, tp.error_feedback, d);
                quads_to_adjacent(d, w3);
            }
            {
                // two runs together (four independent chains per step)
                float v[64];
                __syncwarp();
                tmem_ld64(lb + kYxAccY + 32 * c0, v);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(yfree);
                wait_yp();
                if (!ok) break;
                if (third) tmem_st16(yp + 16 * (c0 + 2), w3);
                uint32_t d0[16], d1[16], w[16];
                narrow64_quads<S>(v, tp.inv_scale, tp.error_feedback, d0, d1);
                quads_to_adjacent(d0, w);
                tmem_st16(yp + 16 * c0, w);
                quads_to_adjacent(d1, w);
                tmem_st16(yp + 16 * (c0 + 1), w);
            }
            tmem_st_wait();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&ypacked[tl & 1]);
        }
    } else if (warp >= 2 + kYxConvWarps && warp < kYxXWarp) {
        // Epilogue: x accumulator -> re-illumination -> next field / final outputs.
        const int ew = warp - 2 - kYxConvWarps;
        const int quad = warp & 3, part = ew >> 2;  // part: x-outputs part * 64 .. + 64 of the tile
        const uint32_t lb = tmem + ((uint32_t) (quad * 32) << 16);
        uint8_t *stg = stage_out + ew * 2 * kXStageWarpBytes;
        typename Sched::Cursor cur;
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const YxTile t = sched.tile(g, &tmap, &omap, cur);
            const int prow = yx_out_perm(lane);  // this lane's y-output within the quadrant
            const int64_t y = t.y0 + quad * 32 + prow;
            const bool live_row = y < t.ny;
            const int64_t row = (int64_t) t.z * t.ny + y;
            MaskWords mw[2] = {};
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const int64_t xb = t.x0 + part * 64 + 32 * k;
                if (live_row && xb < t.nx)
                    mw[k] = load_mask_words<FMT>(t.mask, row * t.nx + xb, t.nx - xb < 32 ? (int) (t.nx - xb) : 32,
                                                 t.n_vox);
            }
            if (!__all_sync(0xffffffffu, mbar_wait(xfull, (uint32_t) (tl & 1), 2))) break;
            tc_fence_after();
            // Both runs read at once, so the x accumulator is free for x(tl + 1)
            // before this warp's rounding and stores.
            float h[64];
            tmem_ld64(lb + kYxAccX + part * 64, h);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(xempty);
            const uint32_t m0 = mask_flags<FMT>(mw[0], t.mask), m1 = mask_flags<FMT>(mw[1], t.mask);
            if (FINAL) {
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    const int64_t xb = t.x0 + part * 64 + 32 * k;
                    float hk[32];  // x order
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        hk[j] = h[32 * k + 2 * j];
                        hk[16 + j] = h[32 * k + 2 * j + 1];
                    }
                    contig_final32(hk, k ? m1 : m0, live_row ? row : t.rows, t.rows, t.nx, xb, tp.inv_scale,
                                   t.out_u16, t.field_out);
                }
            } else {
                // Both runs rounded together (two independent chains per step),
                // then one TMA store per run of the warp's 32 rows x 32 voxels
                // (64-byte swizzle of the store map, which clips rows and columns
                // outside the volume) from the warp's two staging buffers.  The
                // tile's stores form one bulk group, so the wait covers the
                // previous tile's stores, the last readers of both buffers.
                uint32_t dd[2][16];
                narrow64_pairs_forced_adjacent<S>(h, tp.inv_scale, tp.error_feedback, m0, m1, dd[0], dd[1]);
                if (lane == 0) bulk_wait_read<0>();
                __syncwarp();
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    uint32_t q[16];
                    pairs_to_adjacent(dd[k], q);
                    uint8_t *sb = stg + k * kXStageWarpBytes;
#pragma unroll
                    for (int i = 0; i < 4; i++)
                        *reinterpret_cast<uint4 *>(sb + prow * 64 + ((i ^ ((prow >> 1) & 3)) << 4)) =
                            make_uint4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
                }
                fence_proxy_async_smem();
                __syncwarp();
                if (lane == 0) {
                    const int yq = t.y0 + quad * 32;
#pragma unroll
                    for (int k = 0; k < 2; k++) {
                        const int64_t xb = t.x0 + part * 64 + 32 * k;
                        if (xb < t.nx && yq < t.ny) {
                            uint8_t *sb = stg + k * kXStageWarpBytes;
                            if (t.rows_yzx) tma_store_3d(t.out, sb, (int) xb, t.z, yq);
                            else tma_store_3d(t.out, sb, (int) xb, yq, t.z);
                        }
                    }
                    bulk_commit();
                }
            }
        }
        if (!FINAL && lane == 0) bulk_wait_all();
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kYxTmemCols);
    }
}

}  // namespace tc
}  // namespace maxi
