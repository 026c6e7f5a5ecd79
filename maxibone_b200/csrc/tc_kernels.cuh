// Tensor-core (tcgen05) pass kernels for 16-bit field storage (BF16 / FP16),
// shared by the single-volume passes (tc_pass.cu) and the multi-volume
// persistent passes (tc_batch.cu).  A kernel is written once against a
// "schedule" that maps the launch's global work index to one volume's column
// (z / y passes) or tile (x pass): OneVolume* for a single volume whose tensor
// maps are kernel parameters, ManyVolumes* for a device table of volumes
// searched through prefix sums.  Both forms run the same instructions on a
// given tile, so a batch reproduces the single-volume results bit for bit.
//
// z / y passes.  A 1-D convolution along an axis is a banded Toeplitz matrix
// product.  For a tile of 128 consecutive outputs along the axis and TN
// x-columns:
//
//     D[o, x] = sum_j T[o, j] * F[a0 - R + j, x],   T[o, j] = k[j - o] for 0 <= j - o <= 2R
//
// M = 128 outputs (TMEM lanes), N = TN x-columns (TMEM columns), K = KP >=
// 128 + 2R input rows.  T is written once per CTA into tensor memory (the A
// operand of tcgen05.mma may live there: row o in lane o, K packed two per
// column), so the MMAs read only the field tile from shared memory -- with
// both operands in shared memory the MMAs' operand reads, not HBM, set the
// pass time.  The field tile F arrives by TMA (x contiguous: MN-major,
// 128-byte swizzle; rows outside the volume are zero-filled by TMA, which is
// exactly the reference's zero boundary).  Coefficients are split into a high
// and a low 16-bit part (T = T_hi + T_lo, two MMAs into one FP32 accumulator)
// so the effective kernel keeps ~16 significant bits and its sum stays 1 to
// ~1e-6: with single-rounded 16-bit coefficients the kernel's gain error
// compounds over 3 x R passes.  FP16 coefficients are scaled by 2^10 to stay in
// the normal range; the epilogue undoes the scale exactly.  With hi_only the
// passes use one 16-bit set instead, each tap rounded up or down at a searched
// scale (undone by the epilogue like FP16's) so that the set keeps the kernel's
// sum and second moment (tc_round_taps_scaled): one MMA per K step instead of
// two, half the passes' tensor-core work.
//
// Row order of the 16-bit field between repetitions.  The z pass is the only
// pass whose tile rows lie on different planes: read from the [z][y][x] volume
// every row of its 64 x KP box comes from another plane, and TMA delivers such
// boxes at well under the rate of the y pass's boxes (rows one x-row apart).
// So the x pass (which writes whole rows and can put them anywhere) stores
// the field of every repetition but the last with its rows in [y][z][x] order,
// and the next z pass reads its columns as rows nx apart, like the y pass.
// The z pass writes [z][y][x] again; the first repetition's z pass reads the
// initial [z][y][x] field.
//
// x pass.  The field is the A operand: 128 volume rows (M, TMEM lanes) x 128
// x-outputs, so each epilogue thread owns 32 consecutive voxels of one row --
// the layout re-illumination, error feedback along x and vector stores want.
// D[r, o] = sum_j F[r, x0 - RA + j] * Tt[j, o] with RA = R rounded up to 8 (TMA
// x coordinates must be 16-byte aligned); Tt[j, o] = k[j - o - RA + R].  The
// high and low coefficient halves sit in one K-major operand (rows 0..127
// Tt_hi, 128..255 Tt_lo); two N = 128 MMAs accumulate both into the same FP32
// accumulator, so the epilogue reads one value per voxel.
//
// Warp roles in a persistent CTA (one per SM): warp 0 issues TMA loads into a
// tile ring (and L2 prefetches a few tiles ahead), warp 1 issues the MMAs (one
// thread) into a double-buffered TMEM accumulator, the other warps (8 in the
// z / y passes, 16 in the x pass) drain TMEM (tcgen05.ld), narrow to the
// storage type and store.  With error feedback on,
// the rounding error of each stored value is carried to its x-neighbour
// (chains of 16 voxels along x, two of them advancing together): the stored
// field's rounding noise becomes high-pass along x and the next x pass
// removes it.  Every wait is bounded:
// on a timeout the kernel records a code in g_tc_error and winds down, the
// producer first letting the copies it started land and the MMA issuer its
// MMAs complete (both bounded), so no asynchronous write outlives the CTA.
#pragma once

#include <cudaTypedefs.h>

#include "host_util.h"
#include "tc_batch.h"
#include "tc_common.cuh"
#include "tc_pass.h"

namespace maxi {
namespace tc {

constexpr int kTM = 128;      // outputs along the axis (z / y) or rows (x) per tile
constexpr int kXTN = 128;     // x outputs per x-pass tile
constexpr int kXStages = 2;   // TMA ring depth of the x pass
constexpr int kPrefetch = 3;  // tiles prefetched into L2 ahead of the ring
// L2 prefetch depth of the z / y passes (0: none; their TMA ring alone keeps
// enough loads in flight).  Measured per 1024^3 BF16 z pass: 0.80 ms with
// none, 0.85 with 1 tile, 0.86 with 2, 0.88 with 3, 1.04 with 6.
constexpr int kPrefetchStrided = 0;
constexpr int kEpiWarps = 8;  // z / y passes: two warps per TMEM lane quadrant, each drains half the columns
constexpr int kThreads = 64 + 32 * kEpiWarps;  // warp 0 TMA, warp 1 MMA, warps 2..9 epilogue
// The x pass's epilogue (mask, re-illumination, error feedback, stores) is the
// longest: four warps per lane quadrant, each drains 32 of the 128 columns.
constexpr int kXEpiWarps = 16;
constexpr int kXThreads = 64 + 32 * kXEpiWarps;  // warp 0 TMA, warp 1 MMA, warps 2..17 epilogue

// z / y passes: 128-column tiles (64 for radius > 64) in a 3-deep ring.  The
// z pass stages its stores so one instruction writes 8 rows (its output rows
// lie on different planes); the y pass writes each warp's 32 x 32 chunks with
// TMA bulk stores.  Batches (radius <= 32) always use 128-column tiles.
template <bool AXIS_Z> struct StridedShape {
    static constexpr int kTN = 128;
    static constexpr int kStages = 3;
};
constexpr int kStridedStages = 3;
__host__ __device__ constexpr int strided_tn(int radius) { return radius <= 64 ? 128 : 64; }

// Tensor memory of the strided passes (512 columns): accumulators [0, 2 TN),
// then the Toeplitz halves, kcols columns each (K / 2 rounded up to 32: 96 up
// to radius 32, 128 up to 64, 192 up to 128).
constexpr uint32_t kTmemColsStrided = 512;
__host__ __device__ constexpr int toeplitz_cols(int kp) { return ((kp / 2) + 31) / 32 * 32; }

// Per-epilogue-warp staging: two 32-row x 32-column 16-bit buffers, 64-byte
// rows with their 16-byte chunks XOR-swizzled by row / 2 (the y pass's store
// map uses the same 64-byte swizzle; the z pass reads the rows back itself).
constexpr int kStageWarpBytes = 2 * 32 * 64;

__host__ __device__ constexpr int strided_smem_bytes(int kp, int tn, int stages) {
    return 1024 /*alignment slack*/ + stages * (tn / 64) * kp * 128 /*B ring*/ + 1024 /*barriers, TMEM slot*/ +
           kEpiWarps * kStageWarpBytes;
}

// x-pass staging of one epilogue warp's 32 rows x 32 columns of 16-bit output
// (64-byte rows, 16-byte chunks XOR-swizzled by row / 2).
constexpr int kXStageWarpBytes = 32 * 64;

__host__ __device__ constexpr int contig_smem_bytes_tc(int kp, int kpa) {
    return 1024 + kpa * 2 * kXTN * 2 /*Tt_hi|Tt_lo, 256 rows*/ + kXStages * (kpa / 64) * kTM * 128 /*A ring*/ +
           1024 /*barriers, TMEM slot*/ + kXEpiWarps * kXStageWarpBytes;
}

// Taps and K extents of one pass.  K rows longer than a TMA box (256) are
// loaded as nbox boxes of box_rows rows.
struct PassTaps {
    int radius, ra, kp, kpa;  // radius, x-pass left pad, K (multiple of 16), K rounded to 64
    int kcols, nbox, box_rows;
    int error_feedback;
    int hi_only;  // one coefficient set (hi, rounded to keep the kernel's sum and second moment), no lo MMAs
    float inv_scale;
    uint16_t hi[2 * kTcMaxRadiusWide + 1];
    uint16_t lo[2 * kTcMaxRadiusWide + 1];
};

// One column of a z / y pass: n_at axis tiles of TN x-columns at (x0, oth).
// in_rows: the load map is over (x, axis, other) -- the y pass, and the z pass
// reading [y][z][x] rows -- instead of the z pass's (x, y, z).
struct StridedCol {
    const CUtensorMap *in;       // load map (box 64 x KP along the axis)
    const CUtensorMap *out_map;  // y pass: store map (box 32 x 32, 64-byte swizzle)
    void *out;
    int64_t A, stride_a, stride_o, nx;
    int n_at, x0, oth, in_rows;
};

// One tile of the x pass: 128 rows from r0, 128 x-outputs from x0.  Rows are
// numbered z * ny + y.  out_nz > 0: the storage-type output goes to [y][z][x]
// rows of a volume of out_nz planes, at plane out_z0 + z.
struct ContigTile {
    const CUtensorMap *in;       // load map (box 64 x 128 rows)
    const void *mask;
    uint16_t *out;               // storage-type field (not final)
    uint16_t *out_u16;           // final
    float *field_out;            // final, optional
    int64_t rows, nx, r0;
    int64_t ny, out_nz, out_z0;
    int x0;
};

// Element index of row `row` (z * ny + y), column x in the x pass's
// storage-type output.
// Row and tile counts stay below 2^32 (tc_supported), so the divisions here
// and in the schedules are 32-bit.
__device__ __forceinline__ int64_t contig_out_index(const ContigTile &t, int64_t row, int64_t x) {
    if (t.out_nz == 0) return row * t.nx + x;
    const uint32_t ny = (uint32_t) t.ny, z = (uint32_t) row / ny, y = (uint32_t) row - z * ny;
    return (((int64_t) y * t.out_nz + t.out_z0 + z) * t.nx) + x;
}

__device__ __forceinline__ int find_volume(const int64_t *prefix, int n_vol, int64_t g) {
    int lo = 0, hi = n_vol - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(prefix + mid) <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Mask flags of up to 32 voxels of a row in two steps: load_mask_words issues
// the loads (bit-packed: the one or two words the voxels span), mask_flags
// turns them into bit q = voxel q.  uint8 masks are read in mask_flags.
struct MaskWords {
    uint32_t hi = 0, lo = 0;
    int64_t idx = 0, n = 0;
    int shift = 0, count = 0;  // count 0: no voxels
};

template <int FMT>
__device__ __forceinline__ MaskWords load_mask_words(const void *m, int64_t idx, int count, int64_t n) {
    MaskWords w;
    w.idx = idx;
    w.count = count;
    w.n = n;
    if (FMT == MAXI_MASK_BITPACKED) {
        const uint32_t *p = static_cast<const uint32_t *>(m);
        const int64_t w0 = idx >> 5;
        w.shift = (int) (idx & 31);
        w.hi = __ldg(p + w0);
        w.lo = (w.shift > 0 && (w0 + 1) * 32 < n) ? __ldg(p + w0 + 1) : 0u;
    }
    return w;
}

template <int FMT>
__device__ __forceinline__ uint32_t mask_flags(const MaskWords &w, const void *m) {
    if (w.count == 0) return 0u;
    if (FMT == MAXI_MASK_BITPACKED) {
        const uint32_t msb_first = (uint32_t) (((((uint64_t) w.hi << 32) | w.lo) << w.shift) >> 32);  // voxel idx at bit 31
        const uint32_t r = __brev(msb_first);                                                          // voxel idx at bit 0
        return w.count >= 32 ? r : (r & ((1u << w.count) - 1u));
    }
    return row_mask32<FMT>(m, w.idx, w.count, w.n);
}

// ---- schedules -------------------------------------------------------------------

// Each role of a kernel walks the launch's work indices in increasing order
// and keeps a Cursor (the volume it is in and that volume's index range), so
// the binary search over the volumes runs only when the walk leaves the
// current volume.
struct OneVolumeStrided {
    static constexpr bool kParamMaps = true;
    struct Cursor {};
    void *out;
    int64_t A, nx, stride_a, stride_o;
    int n_at, n_xc, tn, in_rows;
    int64_t n_cols;
    __device__ __forceinline__ int64_t total() const { return n_cols; }
    __device__ __forceinline__ StridedCol col(int64_t g, const CUtensorMap *in, const CUtensorMap *out_map,
                                              Cursor &) const {
        StridedCol c;
        c.in = in;
        c.out_map = out_map;
        c.out = out;
        c.A = A;
        c.stride_a = stride_a;
        c.stride_o = stride_o;
        c.nx = nx;
        c.n_at = n_at;
        c.oth = (int) ((uint32_t) g / (uint32_t) n_xc);
        c.x0 = ((int) g - c.oth * n_xc) * tn;
        c.in_rows = in_rows;
        return c;
    }
};

struct ManyVolumesStrided {
    static constexpr bool kParamMaps = false;
    const TcVol *vols;
    const int64_t *prefix;  // n_vol + 1 prefix sums of the volumes' columns
    int n_vol, axis_z, in_buf, tn, z_in_rows;  // z_in_rows: the z pass reads [y][z][x] rows
    // The z / y kernels have registers to spare: the cursor keeps the current
    // volume's column data, so a column within it costs no table reads.
    struct Cursor {
        int64_t lo = 0, hi = 0;  // the current volume's columns [lo, hi)
        int n_xc = 1;
        StridedCol base;
    };
    __device__ __forceinline__ int64_t total() const { return __ldg(prefix + n_vol); }
    __device__ __forceinline__ StridedCol col(int64_t g, const CUtensorMap *, const CUtensorMap *, Cursor &cur) const {
        if (g < cur.lo || g >= cur.hi) {
            const int v = find_volume(prefix, n_vol, g);
            const TcVol &vol = vols[v];
            cur.lo = __ldg(prefix + v);
            cur.hi = __ldg(prefix + v + 1);
            cur.n_xc = axis_z ? vol.n_xc_z : vol.n_xc_y;
            StridedCol &c = cur.base;
            c.in = axis_z ? (z_in_rows ? &vol.zrows[in_buf] : &vol.map[0][in_buf]) : &vol.map[1][in_buf];
            c.in_rows = axis_z ? z_in_rows : 1;
            c.out_map = &vol.ystore[in_buf ^ 1];
            c.out = vol.buf[in_buf ^ 1];
            c.A = axis_z ? vol.nz : vol.ny;
            c.stride_a = axis_z ? vol.ny * vol.nx : vol.nx;
            c.stride_o = axis_z ? vol.nx : vol.ny * vol.nx;
            c.nx = vol.nx;
            c.n_at = axis_z ? vol.n_at_z : vol.n_at_y;
        }
        const int64_t local = g - cur.lo;
        StridedCol c = cur.base;
        c.oth = (int) ((uint32_t) local / (uint32_t) cur.n_xc);
        c.x0 = ((int) local - c.oth * cur.n_xc) * tn;
        return c;
    }
};

struct OneVolumeContig {
    static constexpr bool kParamMaps = true;
    struct Cursor {};
    const void *mask;
    void *out;
    uint16_t *out_u16;
    float *field_out;
    int64_t rows, nx, ny, out_nz, out_z0;
    int n_xt;
    int64_t n_tiles;
    __device__ __forceinline__ int64_t total() const { return n_tiles; }
    __device__ __forceinline__ ContigTile tile(int64_t g, const CUtensorMap *in, Cursor &) const {
        ContigTile t;
        t.in = in;
        t.mask = mask;
        t.out = static_cast<uint16_t *>(out);
        t.out_u16 = out_u16;
        t.field_out = field_out;
        t.rows = rows;
        t.nx = nx;
        t.ny = ny;
        t.out_nz = out_nz;
        t.out_z0 = out_z0;
        const uint32_t rt = (uint32_t) g / (uint32_t) n_xt;
        t.r0 = (int64_t) rt * kTM;
        t.x0 = ((int) g - (int) rt * n_xt) * kXTN;
        return t;
    }
};

struct ManyVolumesContig {
    static constexpr bool kParamMaps = false;
    const TcVol *vols;
    const int64_t *prefix;  // n_vol + 1 prefix sums of the volumes' x tiles
    int n_vol, in_buf, out_rows;  // out_rows: the storage output goes to [y][z][x] rows
    struct Cursor {
        int64_t lo = 0, hi = 0;  // the current volume's tiles [lo, hi)
        int v = 0;
    };
    __device__ __forceinline__ int64_t total() const { return __ldg(prefix + n_vol); }
    __device__ __forceinline__ ContigTile tile(int64_t g, const CUtensorMap *, Cursor &cur) const {
        if (g < cur.lo || g >= cur.hi) {
            cur.v = find_volume(prefix, n_vol, g);
            cur.lo = __ldg(prefix + cur.v);
            cur.hi = __ldg(prefix + cur.v + 1);
        }
        const TcVol &vol = vols[cur.v];
        const int64_t local = g - cur.lo;
        ContigTile t;
        t.in = &vol.map[2][in_buf];
        t.mask = vol.mask;
        t.out = static_cast<uint16_t *>(vol.buf[in_buf ^ 1]);
        t.out_u16 = vol.out_u16;
        t.field_out = vol.field_out;
        t.rows = vol.nz * vol.ny;
        t.nx = vol.nx;
        t.ny = vol.ny;
        t.out_nz = out_rows ? vol.nz : 0;
        t.out_z0 = 0;
        const uint32_t rt = (uint32_t) local / (uint32_t) vol.n_xt;
        t.r0 = (int64_t) rt * kTM;
        t.x0 = ((int) local - (int) rt * vol.n_xt) * kXTN;
        return t;
    }
};

template <class Sched> struct StridedLaunch {
    Sched sched;
    PassTaps taps;
};

template <class Sched> struct ContigLaunch {
    Sched sched;
    PassTaps taps;
    int final_pass;
};

// ---- z / y passes ------------------------------------------------------------------

template <typename S, bool AXIS_Z, int TN, class Sched>
__global__ void __launch_bounds__(kThreads, 1)
tc_strided_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmap_out,
                  const __grid_constant__ StridedLaunch<Sched> p) {
    constexpr int STAGES = kStridedStages, CHUNKS = TN / 64;
    const PassTaps &tp = p.taps;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *ring = smem_raw + (((raw + 1023) & ~1023u) - raw);
    const int stage_bytes = CHUNKS * tp.kp * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + STAGES * stage_bytes);
    uint64_t *full = bars, *empty = bars + STAGES, *tfull = bars + 2 * STAGES, *tempty = bars + 2 * STAGES + 2;
    uint64_t *drain = bars + 2 * STAGES + 4;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 5);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;  // 1024-byte aligned
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = p.sched.total();

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kEpiWarps); }
        mbar_init(drain, 1);
        fence_barrier_init();
        if (Sched::kParamMaps) prefetch_tmap(&tmap);
    }
    __syncwarp();
    if (warp == 0) {
        tmem_alloc(tmem_slot, kTmemColsStrided);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp >= 2) {
        // Toeplitz halves into tensor memory, zero outside the band: the two
        // warps of a lane quadrant write T_hi and T_lo of its 32 rows.
        const int quad = warp & 3, lo_half = (warp - 2) >> 2;
        const int o = quad * 32 + lane;
        const uint16_t *taps = lo_half ? tp.lo : tp.hi;
        for (int ch = 0; ch < tp.kcols / 32; ch++) {
            uint32_t r[32];
#pragma unroll
            for (int j = 0; j < 32; j++) {
                uint32_t v = 0;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int k = 2 * (ch * 32 + j) + e, t = k - o;
                    if (t >= 0 && t <= 2 * tp.radius && k < tp.kp) v |= (uint32_t) taps[t] << (16 * e);
                }
                r[j] = v;
            }
            tmem_st32(tmem + ((uint32_t) (quad * 32) << 16) + 2 * TN + (lo_half ? tp.kcols : 0) + ch * 32, r);
        }
        tmem_st_wait();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 0 && lane == 0) {
        // TMA producer; L2 prefetch kPrefetch tiles ahead, into this CTA's next column.
        int64_t tl = 0;
        bool ok = true;
        int64_t g = blockIdx.x;
        typename Sched::Cursor cc;
        StridedCol cur = p.sched.col(g < total ? g : 0, &tmap, &tmap_out, cc), nxt = cur;
        for (; ok && g < total; g += gridDim.x) {
            const bool has_next = g + gridDim.x < total;
            if (has_next) nxt = p.sched.col(g + gridDim.x, &tmap, &tmap_out, cc);
            for (int at = 0; at < cur.n_at; at++, tl++) {
                const int s = (int) (tl % STAGES);
                const uint32_t ph = (uint32_t) ((tl / STAGES) & 1);
                if (!mbar_wait(&empty[s], ph ^ 1, 1)) { ok = false; break; }
                if (kPrefetchStrided > 0) {
                    const int ap = at + kPrefetchStrided;
                    const CUtensorMap *pm = nullptr;
                    int px = 0, po = 0, pa = 0, pr = 0;
                    if (ap < cur.n_at) { pm = cur.in; px = cur.x0; po = cur.oth; pa = ap; pr = cur.in_rows; }
                    else if (has_next && ap - cur.n_at < nxt.n_at) {
                        pm = nxt.in; px = nxt.x0; po = nxt.oth; pa = ap - cur.n_at; pr = nxt.in_rows;
                    }
                    if (pm) {
                        for (int c = 0; c < CHUNKS; c++)
                            for (int b = 0; b < tp.nbox; b++) {
                                const int a = pa * kTM - tp.radius + b * tp.box_rows;
                                if (pr) tma_prefetch_3d(pm, px + 64 * c, a, po);
                                else tma_prefetch_3d(pm, px + 64 * c, po, a);
                            }
                    }
                }
                const int a_in = at * kTM - tp.radius;
                mbar_arrive_expect_tx(&full[s], stage_bytes);
                for (int c = 0; c < CHUNKS; c++)
                    for (int b = 0; b < tp.nbox; b++) {
                        uint8_t *dst = ring + s * stage_bytes + c * tp.kp * 128 + b * tp.box_rows * 128;
                        const int a = a_in + b * tp.box_rows;
                        if (cur.in_rows) tma_load_3d(dst, cur.in, cur.x0 + 64 * c, a, cur.oth, &full[s]);
                        else tma_load_3d(dst, cur.in, cur.x0 + 64 * c, cur.oth, a, &full[s]);
                    }
            }
            cur = nxt;
        }
        // The copies this thread started land before the CTA can exit (the last
        // use of each ring stage; bounded, so an aborted run still ends).
        for (int64_t k = tl - STAGES; k < tl; k++)
            if (k >= 0) mbar_wait(&full[k % STAGES], (uint32_t) ((k / STAGES) & 1), 1);
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc = idesc_f16(fmt, 0 /*A K-major*/, 1 /*B MN-major*/, kTM, TN);
        const uint32_t b0 = smem_u32(ring);
        int64_t tl = 0;
        bool ok = true;
        typename Sched::Cursor cc;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x) {
            const int n_at = p.sched.col(g, &tmap, &tmap_out, cc).n_at;
            for (int at = 0; at < n_at; at++, tl++) {
                const int s = (int) (tl % STAGES);
                const uint32_t ph = (uint32_t) ((tl / STAGES) & 1);
                const int d = (int) (tl & 1);
                const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
                if (!mbar_wait(&full[s], ph, 1) || !mbar_wait(&tempty[d], dph ^ 1, 3)) { ok = false; break; }
                tc_fence_after();
                const uint32_t dt = tmem + d * TN;
                // K step ks: 16 rows of the field tile (2048 bytes on, i.e. +128 in the
                // descriptor's address field) and 8 tensor-memory columns of T.
                const uint64_t bd = smem_desc_sw128(b0 + s * stage_bytes, tp.kp * 128, 1024);
                const uint32_t a_hi = tmem + 2 * TN, a_lo = a_hi + tp.kcols;
                for (int ks = 0; ks < tp.kp / 16; ks++) {
                    umma_f16_ts(dt, a_hi + ks * 8, bd + (uint64_t) (ks * 128), idesc, ks > 0 ? 1u : 0u);
                    if (!tp.hi_only) umma_f16_ts(dt, a_lo + ks * 8, bd + (uint64_t) (ks * 128), idesc, 1u);
                }
                umma_commit(&empty[s]);
                umma_commit(&tfull[d]);
            }
        }
        // Every MMA this thread issued completes before the CTA winds down.
        umma_commit(drain);
        mbar_wait(drain, 0, 2);
    } else if (warp >= 2) {
        // Epilogue: TMEM -> registers -> storage type -> global.
        const int quad = warp & 3;           // TMEM lane quadrant this warp may access
        const int half = (warp - 2) >> 2;    // which half of the columns it drains
        uint8_t *stg = stage_out + (warp - 2) * kStageWarpBytes;
        int sbuf = 0;
        int64_t tl = 0;
        bool ok = true;
        typename Sched::Cursor cc;
        for (int64_t g = blockIdx.x; ok && g < total; g += gridDim.x) {
            const StridedCol c = p.sched.col(g, &tmap, &tmap_out, cc);
            S *out = static_cast<S *>(c.out);
            for (int at = 0; at < c.n_at; at++, tl++) {
                const int d = (int) (tl & 1);
                const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
                if (!mbar_wait(&tfull[d], dph, 2)) { ok = false; break; }
                tc_fence_after();
                const int c0 = half * CHUNKS;  // this warp's 32-column chunks
                const uint32_t tbase = tmem + ((uint32_t) (quad * 32) << 16) + d * TN;
#pragma unroll
                for (int cc = 0; cc < CHUNKS; cc++) {
                    float va[32];
                    __syncwarp();
                    tmem_ld32(tbase + (c0 + cc) * 32, va);
                    uint32_t qd[16], q[16];  // q[i]: voxels 2i, 2i + 1
                    narrow32_pairs<S, false>(va, tp.inv_scale, tp.error_feedback, 0u, 0xffffffffu, qd);
                    pairs_to_adjacent(qd, q);
                    const int64_t xb = (int64_t) c.x0 + (c0 + cc) * 32;
                    if (AXIS_Z) {
                        // z pass: lanes' rows lie on different planes (2 MB apart at 1024^2);
                        // stage the 32 x 32 chunk and write 8 rows (8 x 64 bytes) per instruction.
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
                            const int64_t ar = (int64_t) at * kTM + quad * 32 + rr;
                            const uint4 w = *reinterpret_cast<const uint4 *>(stg + rr * 64 + ((sub ^ ((rr >> 1) & 3)) << 4));
                            if (ar < c.A && xb + sub * 8 < c.nx)
                                *reinterpret_cast<uint4 *>(out + ar * c.stride_a + (int64_t) c.oth * c.stride_o + xb +
                                                           sub * 8) = w;
                        }
                    } else {
                        // y pass: TMA store of the warp's 32 rows x 32 columns (64-byte swizzle of
                        // the store map; the map clips rows and columns outside the volume).
                        if (lane == 0) bulk_wait_read<1>();  // the store issued two chunks ago has read this buffer
                        __syncwarp();
                        uint8_t *sb = stg + sbuf * 2048;
#pragma unroll
                        for (int i = 0; i < 4; i++)
                            *reinterpret_cast<uint4 *>(sb + lane * 64 + ((i ^ ((lane >> 1) & 3)) << 4)) =
                                make_uint4(q[4 * i], q[4 * i + 1], q[4 * i + 2], q[4 * i + 3]);
                        fence_proxy_async_smem();
                        __syncwarp();
                        // Every chunk commits exactly one bulk group (an empty one when the
                        // chunk lies outside the volume), so that bulk_wait_read<1> above always
                        // covers the store that last read the buffer being refilled.
                        if (lane == 0) {
                            if (xb < c.nx && at * kTM + quad * 32 < c.A)
                                tma_store_3d(c.out_map, sb, (int) xb, at * kTM + quad * 32, c.oth);
                            bulk_commit();
                        }
                        sbuf ^= 1;
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[d]);
            }
        }
    }
    if (!AXIS_Z && warp >= 2 && lane == 0) bulk_wait_all();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemColsStrided);
    }
}

// ---- x pass ------------------------------------------------------------------------

template <typename S, int FMT, class Sched>
__global__ void __launch_bounds__(kXThreads, 1)
tc_contig_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ ContigLaunch<Sched> p) {
    const PassTaps &tp = p.taps;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *smem = smem_raw + (((raw + 1023) & ~1023u) - raw);
    uint8_t *tt = smem;                                  // K-major, 256 rows (hi 0..127, lo 128..255)
    uint8_t *ring = tt + tp.kpa * 2 * kXTN * 2;
    const int nkb = tp.kpa / 64;                         // 64-wide x boxes per stage
    const int stage_bytes = nkb * kTM * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kXStages * stage_bytes);
    uint64_t *full = bars, *empty = bars + kXStages, *tfull = bars + 2 * kXStages, *tempty = bars + 2 * kXStages + 2;
    uint64_t *drain = bars + 2 * kXStages + 4;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kXStages + 5);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = p.sched.total();

    for (int e = threadIdx.x; e < 2 * kXTN * tp.kpa; e += kXThreads) {
        const int n = e / tp.kpa, j = e - n * tp.kpa;
        const int o = n & (kXTN - 1);
        const int t = j - o - tp.ra + tp.radius;  // tap index 0..2R
        uint16_t v = 0;
        if (t >= 0 && t <= 2 * tp.radius && j < tp.kp) v = n < kXTN ? tp.hi[t] : tp.lo[t];
        *reinterpret_cast<uint16_t *>(tt + sw128_kmajor_offset(n, j, 2 * kXTN)) = v;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kXStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kXEpiWarps); }
        mbar_init(drain, 1);
        fence_barrier_init();
        if (Sched::kParamMaps) prefetch_tmap(&tmap);
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
        typename Sched::Cursor cc, cp;  // current tile, L2-prefetched tile
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int s = (int) (tl % kXStages);
            const uint32_t ph = (uint32_t) ((tl / kXStages) & 1);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) break;
            const int64_t gp = g + kPrefetch * (int64_t) gridDim.x;
            if (gp < total) {
                const ContigTile t = p.sched.tile(gp, &tmap, cp);
                for (int kb = 0; kb < nkb; kb++) tma_prefetch_3d(t.in, t.x0 - tp.ra + 64 * kb, (int) t.r0, 0);
            }
            const ContigTile t = p.sched.tile(g, &tmap, cc);
            mbar_arrive_expect_tx(&full[s], stage_bytes);
            for (int kb = 0; kb < nkb; kb++)
                tma_load_3d(ring + s * stage_bytes + kb * kTM * 128, t.in, t.x0 - tp.ra + 64 * kb, (int) t.r0, 0, &full[s]);
        }
        for (int64_t k = tl - kXStages; k < tl; k++)  // the started copies land before exit (bounded)
            if (k >= 0) mbar_wait(&full[k % kXStages], (uint32_t) ((k / kXStages) & 1), 1);
    } else if (warp == 1 && lane == 0) {
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc = idesc_f16(fmt, 0 /*A K-major*/, 0 /*B K-major*/, kTM, kXTN);
        const uint32_t a0 = smem_u32(ring), b0 = smem_u32(tt);
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int s = (int) (tl % kXStages);
            const uint32_t ph = (uint32_t) ((tl / kXStages) & 1);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&full[s], ph, 1) || !mbar_wait(&tempty[d], dph ^ 1, 3)) break;
            tc_fence_after();
            const uint32_t dt = tmem + d * kXTN;
            for (int ks = 0; ks < tp.kp / 16; ks++) {
                const uint32_t kin = (ks & 3) * 32;
                const uint64_t ad = smem_desc_sw128(a0 + s * stage_bytes + (ks >> 2) * (kTM * 128) + kin, 16, 1024);
                const uint32_t bhi = b0 + (ks >> 2) * (2 * kXTN * 128) + kin;  // rows 0..127: Tt_hi
                umma_f16(dt, ad, smem_desc_sw128(bhi, 16, 1024), idesc, ks > 0 ? 1u : 0u);
                if (!tp.hi_only)
                    umma_f16(dt, ad, smem_desc_sw128(bhi + kXTN * 128, 16, 1024), idesc, 1u);  // rows 128..255: Tt_lo
            }
            umma_commit(&empty[s]);
            umma_commit(&tfull[d]);
        }
        umma_commit(drain);  // the issued MMAs complete before the CTA winds down (bounded)
        mbar_wait(drain, 0, 2);
    } else if (warp >= 2) {
        const int quad = warp & 3;         // TMEM lane quadrant this warp may access
        const int part = (warp - 2) >> 2;  // which 32 of the 128 columns it drains
        const int r = quad * 32 + lane;
        uint8_t *stg = stage_out + (warp - 2) * kXStageWarpBytes;
        // Mask words of this thread's 32 voxels of a tile (bit-packed masks: the
        // one or two words they span), loaded one tile ahead so that their
        // global-memory latency overlaps the previous tile's work.
        auto mask_words = [&](const ContigTile &t) -> MaskWords {
            const int64_t row = t.r0 + r, xb = t.x0 + part * 32;
            if (row >= t.rows || xb >= t.nx) return MaskWords{};
            return load_mask_words<FMT>(t.mask, row * t.nx + xb, t.nx - xb < 32 ? (int) (t.nx - xb) : 32,
                                        t.rows * t.nx);
        };
        typename Sched::Cursor cc;
        MaskWords mw_next = blockIdx.x < total ? mask_words(p.sched.tile(blockIdx.x, &tmap, cc)) : MaskWords{};
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const ContigTile t = p.sched.tile(g, &tmap, cc);
            const MaskWords mwords = mw_next;
            if (g + gridDim.x < total) mw_next = mask_words(p.sched.tile(g + gridDim.x, &tmap, cc));
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&tfull[d], dph, 2)) break;
            tc_fence_after();
            const int64_t row = t.r0 + r;
            const int64_t xb = t.x0 + part * 32;  // this warp's 32 voxels of the row
            const uint32_t mw = mask_flags<FMT>(mwords, t.mask);
            float h[32];
            __syncwarp();
            tmem_ld32(tmem + ((uint32_t) (quad * 32) << 16) + d * kXTN + part * 32, h);
            if (p.final_pass) {
                contig_final32(h, mw, row, t.rows, t.nx, xb, tp.inv_scale, t.out_u16, t.field_out);
            } else if (xb < t.nx) {  // warp-uniform
                // 16-bit field: narrow with error feedback, stage the warp's 32 x 32
                // chunk and write 8 rows (8 x 64 bytes) per instruction -- in [y][z][x]
                // order the warp's rows lie 2 MB apart at 1024^3.
                uint32_t qd[16], q[16];  // q[i]: voxels 2i, 2i + 1
                narrow32_pairs<S, true>(h, tp.inv_scale, tp.error_feedback, mw, 0xffffffffu, qd);
                pairs_to_adjacent(qd, q);
                const int64_t oi = row < t.rows ? contig_out_index(t, row, xb) : -1;
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
                    const uint4 w = *reinterpret_cast<const uint4 *>(stg + rr * 64 + ((sub ^ ((rr >> 1) & 3)) << 4));
                    if (o >= 0 && xb + sub * 8 < t.nx) *reinterpret_cast<uint4 *>(t.out + o + sub * 8) = w;
                }
            }
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

// ---- x pass, transposed form (radius 33..128) --------------------------------------
//
// With K = 128 + RA + R up to 384 the x pass's Toeplitz no longer fits shared
// memory beside its tile ring, so the roles swap: the Toeplitz is the A
// operand, in tensor memory like the z / y passes' (lane o = x output, K
// packed two per column), and 64 volume rows of the field are the B operand
// (K-major: the rows' x runs, as TMA lands them).  D^T[o, r] = sum_j
// Tt[j, o] F[r, x0 - RA + j], so an epilogue thread owns one x of 32
// consecutive rows: error feedback then runs along the rows (y), and the next
// repetition's y pass removes the high-pass noise it leaves.  The mask words
// of the 32 rows are read one per lane and transposed across the warp.
constexpr int kXtRows = 64;       // rows per tile (N)
constexpr int kXtStages = 3;
constexpr int kXtEpiWarps = 8;    // two per lane quadrant, each drains 32 of the 64 rows
constexpr int kXtThreads = 64 + 32 * kXtEpiWarps;
constexpr int kXtStageWarpBytes = 32 * 64;

__host__ __device__ constexpr int contig_t_smem_bytes(int kpa) {
    return 1024 + kXtStages * (kpa / 64) * kXtRows * 128 /*B ring*/ + 1024 /*barriers, TMEM slot*/ +
           kXtEpiWarps * kXtStageWarpBytes;
}

struct OneVolumeContigT {
    static constexpr bool kParamMaps = true;
    const void *mask;
    void *out;
    uint16_t *out_u16;
    float *field_out;
    int64_t rows, nx, ny, out_nz, out_z0;
    int n_xt;
    int64_t n_tiles;
    __device__ __forceinline__ int64_t total() const { return n_tiles; }
    __device__ __forceinline__ ContigTile tile(int64_t g, const CUtensorMap *in) const {
        ContigTile t;
        t.in = in;
        t.mask = mask;
        t.out = static_cast<uint16_t *>(out);
        t.out_u16 = out_u16;
        t.field_out = field_out;
        t.rows = rows;
        t.nx = nx;
        t.ny = ny;
        t.out_nz = out_nz;
        t.out_z0 = out_z0;
        const uint32_t rt = (uint32_t) g / (uint32_t) n_xt;
        t.r0 = (int64_t) rt * kXtRows;
        t.x0 = ((int) g - (int) rt * n_xt) * kXTN;
        return t;
    }
};

// 32 x 32 bit transpose across a warp: lane i holds row i (bit b = column b)
// on entry, lane b holds column b (bit i = row i) on return.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t w, int lane) {
    const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
    for (int k = 0; k < 5; k++) {
        const int sh = 16 >> k;
        const uint32_t m = masks[k];
        const uint32_t y = __shfl_xor_sync(0xffffffffu, w, sh);
        w = (lane & sh) ? ((w & ~m) | ((y & ~m) >> sh)) : ((w & m) | ((y & m) << sh));
    }
    return w;
}

template <typename S, int FMT>
__global__ void __launch_bounds__(kXtThreads, 1)
tc_contig_t_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ ContigLaunch<OneVolumeContigT> p) {
    const PassTaps &tp = p.taps;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t *ring = smem_raw + (((raw + 1023) & ~1023u) - raw);
    const int nkb = tp.kpa / 64;                       // 64-wide x boxes per stage
    const int stage_bytes = nkb * kXtRows * 128;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kXtStages * stage_bytes);
    uint64_t *full = bars, *empty = bars + kXtStages, *tfull = bars + 2 * kXtStages, *tempty = bars + 2 * kXtStages + 2;
    uint64_t *drain = bars + 2 * kXtStages + 4;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 2 * kXtStages + 5);
    uint8_t *stage_out = reinterpret_cast<uint8_t *>(bars) + 1024;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t total = p.sched.total();
    constexpr uint32_t kAcc = 2 * kXtRows;              // accumulator columns; the Toeplitz halves follow

    if (threadIdx.x == 0) {
        for (int s = 0; s < kXtStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], kXtEpiWarps); }
        mbar_init(drain, 1);
        fence_barrier_init();
        prefetch_tmap(&tmap);
    }
    __syncwarp();
    if (warp == 0) {
        tmem_alloc(tmem_slot, kTmemColsStrided);
        tmem_relinquish();
    }
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    if (warp >= 2) {
        // Tt^T halves into tensor memory: lane o holds x output o, K element j
        // the tap j - o - RA + R (zero outside the band).
        const int quad = warp & 3, lo_half = (warp - 2) >> 2;
        const int o = quad * 32 + lane;
        const uint16_t *taps = lo_half ? tp.lo : tp.hi;
        for (int ch = 0; ch < tp.kcols / 32; ch++) {
            uint32_t r[32];
#pragma unroll
            for (int j = 0; j < 32; j++) {
                uint32_t v = 0;
#pragma unroll
                for (int e = 0; e < 2; e++) {
                    const int k = 2 * (ch * 32 + j) + e, t = k - o - tp.ra + tp.radius;
                    if (t >= 0 && t <= 2 * tp.radius && k < tp.kp) v |= (uint32_t) taps[t] << (16 * e);
                }
                r[j] = v;
            }
            tmem_st32(tmem + ((uint32_t) (quad * 32) << 16) + kAcc + (lo_half ? tp.kcols : 0) + ch * 32, r);
        }
        tmem_st_wait();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 0 && lane == 0) {
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int s = (int) (tl % kXtStages);
            const uint32_t ph = (uint32_t) ((tl / kXtStages) & 1);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) break;
            const int64_t gp = g + kPrefetch * (int64_t) gridDim.x;
            if (gp < total) {
                const ContigTile t = p.sched.tile(gp, &tmap);
                for (int kb = 0; kb < nkb; kb++) tma_prefetch_3d(t.in, t.x0 - tp.ra + 64 * kb, (int) t.r0, 0);
            }
            const ContigTile t = p.sched.tile(g, &tmap);
            mbar_arrive_expect_tx(&full[s], stage_bytes);
            for (int kb = 0; kb < nkb; kb++)
                tma_load_3d(ring + s * stage_bytes + kb * kXtRows * 128, t.in, t.x0 - tp.ra + 64 * kb, (int) t.r0, 0,
                            &full[s]);
        }
        for (int64_t k = tl - kXtStages; k < tl; k++)  // the started copies land before exit (bounded)
            if (k >= 0) mbar_wait(&full[k % kXtStages], (uint32_t) ((k / kXtStages) & 1), 1);
    } else if (warp == 1 && lane == 0) {
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc = idesc_f16(fmt, 0 /*A K-major*/, 0 /*B K-major*/, kTM, kXtRows);
        const uint32_t b0 = smem_u32(ring);
        const uint32_t a_hi = tmem + kAcc, a_lo = a_hi + tp.kcols;
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const int s = (int) (tl % kXtStages);
            const uint32_t ph = (uint32_t) ((tl / kXtStages) & 1);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&full[s], ph, 1) || !mbar_wait(&tempty[d], dph ^ 1, 3)) break;
            tc_fence_after();
            const uint32_t dt = tmem + d * kXtRows;
            for (int ks = 0; ks < tp.kp / 16; ks++) {
                // K step ks: 16 x-inputs = 32 bytes inside a 64-wide box of 64 rows.
                const uint64_t bd = smem_desc_sw128(b0 + s * stage_bytes + (ks >> 2) * (kXtRows * 128) + (ks & 3) * 32, 16,
                                                    1024);
                umma_f16_ts(dt, a_hi + ks * 8, bd, idesc, ks > 0 ? 1u : 0u);
                if (!tp.hi_only) umma_f16_ts(dt, a_lo + ks * 8, bd, idesc, 1u);
            }
            umma_commit(&empty[s]);
            umma_commit(&tfull[d]);
        }
        umma_commit(drain);  // the issued MMAs complete before the CTA winds down (bounded)
        mbar_wait(drain, 0, 2);
    } else if (warp >= 2) {
        const int quad = warp & 3;             // TMEM lane quadrant: x outputs quad * 32 + lane
        const int half = (warp - 2) >> 2;      // rows half * 32 .. + 32 of the tile
        uint8_t *stg = stage_out + (warp - 2) * kXtStageWarpBytes;
        int64_t tl = 0;
        for (int64_t g = blockIdx.x; g < total; g += gridDim.x, tl++) {
            const ContigTile t = p.sched.tile(g, &tmap);
            const int64_t rbase = t.r0 + half * 32;
            const int64_t xq = t.x0 + quad * 32;  // this warp's 32 x outputs
            const bool live = xq < t.nx;          // warp-uniform
            // Lane i reads the mask flags of row rbase + i over the warp's 32 x;
            // the transpose gives lane l the flags of its x over the 32 rows.
            uint32_t mrow = 0;
            if (live && rbase + lane < t.rows)
                mrow = row_mask32<FMT>(t.mask, (rbase + lane) * t.nx + xq, t.nx - xq < 32 ? (int) (t.nx - xq) : 32,
                                       t.rows * t.nx);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&tfull[d], dph, 2)) break;
            tc_fence_after();
            float h[32];
            __syncwarp();
            tmem_ld32(tmem + ((uint32_t) (quad * 32) << 16) + d * kXtRows + half * 32, h);
            const uint32_t m = warp_transpose32(mrow, lane);
            const int64_t x = xq + lane;
            if (p.final_pass) {
                if (live && x < t.nx) {
#pragma unroll
                    for (int i = 0; i < 32; i++) {
                        const int64_t row = rbase + i;
                        if (row < t.rows) {
                            const float v = ((m >> i) & 1u) ? 1.0f : h[i] * tp.inv_scale;
                            if (t.out_u16) t.out_u16[row * t.nx + x] = quantise_u16(v);
                            if (t.field_out) t.field_out[row * t.nx + x] = v;
                        }
                    }
                }
            } else if (live) {
                // 16-bit field, error feedback along the rows; stage the 32 rows x 32 x
                // chunk and write 8 rows (8 x 64 bytes) per instruction.
                uint16_t q[32];
                narrow32_masked<S>(h, m, tp.inv_scale, tp.error_feedback, q);
                const int64_t oi = rbase + lane < t.rows ? contig_out_index(t, rbase + lane, xq) : -1;
                __syncwarp();
#pragma unroll
                for (int i = 0; i < 32; i++)
                    *reinterpret_cast<uint16_t *>(stg + i * 64 + ((((lane >> 3) ^ ((i >> 1) & 3))) << 4) + (lane & 7) * 2) = q[i];
                __syncwarp();
                const int sub = lane & 3, rsub = lane >> 2;
#pragma unroll
                for (int r4 = 0; r4 < 4; r4++) {
                    const int rr = r4 * 8 + rsub;
                    const int64_t o = __shfl_sync(0xffffffffu, oi, rr);
                    const uint4 w = *reinterpret_cast<const uint4 *>(stg + rr * 64 + ((sub ^ ((rr >> 1) & 3)) << 4));
                    if (o >= 0 && xq + sub * 8 < t.nx) *reinterpret_cast<uint4 *>(t.out + o + sub * 8) = w;
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[d]);
        }
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemColsStrided);
    }
}

// Fills the taps of one pass: hi/lo halves of kernel x scale (1 for BF16, 2^10 for FP16).
inline void fill_pass_taps(PassTaps &t, const float *kernel, int radius, int ra, int kp, bool is_bf16,
                           bool error_feedback, bool hi_only = false) {
    t.radius = radius;
    t.ra = ra;
    t.kp = kp;
    t.kpa = (int) round_up(kp, 64);
    t.kcols = toeplitz_cols(kp);
    t.nbox = kp > 256 ? 2 : 1;  // kp is a multiple of 16, so kp / 2 is a whole number of 8-row swizzle atoms
    t.box_rows = kp / t.nbox;
    t.error_feedback = error_feedback ? 1 : 0;
    const float scale = is_bf16 ? 1.0f : 1024.0f;
    t.inv_scale = 1.0f / scale;
    t.hi_only = hi_only ? 1 : 0;
    if (hi_only) {
        t.inv_scale = 1.0f / tc_round_taps_scaled(kernel, radius, is_bf16, scale, t.hi);
        for (int i = 0; i < 2 * radius + 1; i++) t.lo[i] = 0;
    } else {
        tc_split_taps(kernel, radius, is_bf16, scale, t.hi, t.lo);
    }
}

}  // namespace tc
}  // namespace maxi
