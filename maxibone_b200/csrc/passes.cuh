// CUDA-core convolution passes of the diffusion step (sm_100a).
//
// One repetition of the reference step (src/lib/cpp/cpu/diffusion.cc:314-320)
// is three 1-D zero-boundary convolutions -- z, then y, then x -- followed by
// re-illumination of the mask voxels.  Here:
//
//   * strided_pass   : the z and y passes.  The volume is viewed as
//                      [outer][axis][inner] with `inner` contiguous; a CTA stages
//                      a tile of (TA + 2R) axis rows x TI inner columns in shared
//                      memory and each thread produces M consecutive outputs
//                      along the axis for one column.
//   * contig_pass    : the x pass fused with re-illumination (and, on the last
//                      repetition, with the uint16 quantisation).  A CTA stages
//                      32 rows x (TX + 2R) voxels; lane = row, warp = x segment.
//
// Both are register-blocked: each thread reads M + 2R staged values and issues
// M * (2R + 1) FMAs whose coefficients are compile-time indices into the launch
// parameters (constant bank operands), in increasing tap order -- the
// reference's summation order (src/lib/cpp/cpu/diffusion.cc:41-54).  Taps
// outside the volume read zeros, which leave the FP32 sum unchanged, so the
// zero boundary needs no clipping of the tap range.
#pragma once

#include "common.cuh"

namespace maxi {

template <int R> struct Taps { float k[2 * R + 1]; };

// ---- strided (z / y) pass -------------------------------------------------
constexpr int kStrTI = 32;    // inner columns per CTA (one warp wide)
constexpr int kStrTA = 256;   // axis outputs per CTA
constexpr int kStrM = 32;     // axis outputs per thread
constexpr int kStrThreads = kStrTI * (kStrTA / kStrM);  // 256

// The staged tile, or (error-feedback epilogue) the outputs on a 33-word row stride.
template <int R> constexpr int strided_smem_bytes() {
    return ((kStrTA + 2 * R) * kStrTI > kStrTA * (kStrTI + 1) ? (kStrTA + 2 * R) * kStrTI : kStrTA * (kStrTI + 1)) * 4;
}

// EF: error-feedback rounding to the 16-bit storage type along x (the inner
// columns), chains of 16 voxels: the stored rounding noise is high-pass along
// x and the following x pass filters it out.
template <int R, typename S, bool EF = false>
__global__ void __launch_bounds__(kStrThreads)
strided_pass(const S *__restrict__ in, S *__restrict__ out, int64_t A, int64_t I,
             int64_t n_axis_tiles, int64_t n_inner_tiles, const Taps<R> taps) {
    constexpr int ROWS = kStrTA + 2 * R;
    extern __shared__ __align__(16) float s_tile[];  // [ROWS][kStrTI]

    int64_t b = blockIdx.x;
    const int64_t at = b % n_axis_tiles;  b /= n_axis_tiles;   // axis tile fastest: halos hit L2
    const int64_t it = b % n_inner_tiles;
    const int64_t o = b / n_inner_tiles;
    const int64_t a0 = at * kStrTA, i0 = it * kStrTI;
    const int col = threadIdx.x % kStrTI;
    const int seg = threadIdx.x / kStrTI;
    const bool col_ok = i0 + col < I;
    constexpr int VEC = Vec16<S>::N;            // elements per 16-byte chunk
    constexpr int CH = kStrTI / VEC;            // chunks per staged row
    constexpr int RPI = kStrThreads / CH;       // rows staged per iteration
    // Vector path: all columns of the tile inside the volume and 16-byte aligned
    // rows.  Rows outside [0, A) are zero-filled a chunk at a time.
    const bool vec = i0 + kStrTI <= I && I % VEC == 0;
    if (vec) {
        const int chunk = threadIdx.x % CH;
        const int row0 = threadIdx.x / CH;
        const bool rows_inside = a0 >= R && a0 + kStrTA + R <= A;
        const S *src = in + (o * A + a0 - R + row0) * I + i0 + chunk * VEC;
        float *dst = s_tile + row0 * kStrTI + chunk * VEC;
#pragma unroll
        for (int r = row0, k = 0; k < (ROWS + RPI - 1) / RPI; k++, r += RPI) {
            if (ROWS % RPI == 0 || r < ROWS) {
                const int64_t a = a0 - R + r;
                if (rows_inside || (a >= 0 && a < A)) {
                    stage16<S>(dst, src);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; q += 4) *reinterpret_cast<float4 *>(dst + q) = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
            src += RPI * I;
            dst += RPI * kStrTI;
        }
        cp_async_wait_all();
    } else {
        const S *src = in + o * A * I + i0 + col;
        for (int r = seg; r < ROWS; r += kStrThreads / kStrTI) {
            const int64_t a = a0 - R + r;
            float v = 0.0f;
            if (col_ok && a >= 0 && a < A) v = FieldIO<S>::load(src + a * I);
            s_tile[r * kStrTI + col] = v;
        }
    }
    __syncthreads();

    float acc[kStrM];
#pragma unroll
    for (int i = 0; i < kStrM; i++) acc[i] = 0.0f;
    const float *s = s_tile + seg * kStrM * kStrTI + col;
#pragma unroll
    for (int j = 0; j < kStrM + 2 * R; j++) {
        const float v = s[j * kStrTI];
#pragma unroll
        for (int i = 0; i < kStrM; i++) {
            const int t = j - i;
            if (t >= 0 && t <= 2 * R) acc[i] = fmaf(taps.k[t], v, acc[i]);
        }
    }

    if (EF) {
        // Transpose through shared memory: thread -> (axis row, 16 consecutive columns).
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kStrM; i++) s_tile[(seg * kStrM + i) * (kStrTI + 1) + col] = acc[i];
        __syncthreads();
        const int c0 = (threadIdx.x & 1) * 16;
        for (int row = threadIdx.x >> 1; row < kStrTA; row += kStrThreads / 2) {
            const int64_t a = a0 + row;
            if (a >= A) break;
            S *dst = out + (o * A + a) * I + i0 + c0;
            float carry = 0.0f;
#pragma unroll
            for (int c = 0; c < 16; c++) {
                const float w = s_tile[row * (kStrTI + 1) + c0 + c] + carry;
                const S q = FieldIO<S>::narrow(w);
                carry = w - FieldIO<S>::widen(q);
                if (i0 + c0 + c < I) dst[c] = q;
            }
        }
        return;
    }
    if (!col_ok) return;
    S *dst = out + (o * A + a0 + seg * kStrM) * I + i0 + col;
    if (a0 + kStrTA <= A) {
#pragma unroll
        for (int i = 0; i < kStrM; i++, dst += I) *dst = FieldIO<S>::narrow(acc[i]);
    } else {
#pragma unroll
        for (int i = 0; i < kStrM; i++, dst += I)
            if (a0 + seg * kStrM + i < A) *dst = FieldIO<S>::narrow(acc[i]);
    }
}

// ---- contiguous (x) pass + illumination ------------------------------------
constexpr int kConTR = 32;   // rows per CTA (lane = row)
constexpr int kConM = 32;    // x outputs per thread
constexpr int kConWarps = 8;
constexpr int kConTX = kConWarps * kConM;  // 256 x outputs per CTA
constexpr int kConThreads = kConWarps * 32;

template <int R> constexpr int contig_width() { return ((kConTX + 2 * R) + 3) / 4 * 4; }
// Row stride = 4 (mod 32) words: float4 reads by 32 lanes on 32 rows are conflict-free.
template <int R> constexpr int contig_stride() {
    return contig_width<R>() + ((4 - contig_width<R>() % 32) + 32) % 32;
}
template <int R> constexpr int contig_smem_bytes() { return kConTR * contig_stride<R>() * 4; }

// FINAL: last repetition -- write the uint16 output (and optionally the FP32
// field) instead of the storage-type field.
// EF (16-bit storage, not FINAL): the thread's 32 consecutive outputs are
// re-illuminated and rounded with error feedback along x in registers (the
// carry restarts after every mask voxel, which is stored as exactly 1.0).
template <int R, typename S, int MASK_FMT, bool FINAL, bool EF = false>
__global__ void __launch_bounds__(kConThreads, (sizeof(S) == 4 && !FINAL && R <= 32) ? 5 : 1)
contig_pass(const S *__restrict__ in, S *__restrict__ out, const void *__restrict__ mask,
            uint16_t *__restrict__ out_u16, float *__restrict__ field_out,
            int64_t rows, int64_t nx, int64_t n_x_tiles, const Taps<R> taps) {
    constexpr int W = contig_width<R>();
    constexpr int STRIDE = contig_stride<R>();
    constexpr int NJ = (kConM + 2 * R + 3) / 4 * 4;  // staged values read per thread
    extern __shared__ __align__(16) float s_tile[];  // [kConTR][STRIDE]

    const int64_t xt = blockIdx.x % n_x_tiles;
    const int64_t r0 = (blockIdx.x / n_x_tiles) * kConTR;
    const int64_t x0 = xt * kConTX;
    const int tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    constexpr int VEC = Vec16<S>::N;
    // Vector path: full row block, rows and halo start on 16-byte boundaries, and
    // every output pointer aligned for 4-voxel vector access.  Chunks outside
    // [0, nx) are zero-filled (chunks never straddle the row ends).
    const bool vec = r0 + kConTR <= rows && nx % VEC == 0 && R % VEC == 0 &&
                     ((reinterpret_cast<uintptr_t>(out_u16) & 7) | (reinterpret_cast<uintptr_t>(field_out) & 15) |
                      (reinterpret_cast<uintptr_t>(mask) & 3)) == 0;

    if (vec) {
        constexpr int CPR = (kConTX + 2 * R) / VEC;  // chunks per row (exact: R % VEC == 0)
#pragma unroll
        for (int rr = 0; rr < kConTR / kConWarps; rr++) {
            const int r = warp + rr * kConWarps;
            const S *src = in + (r0 + r) * nx + x0 - R;
#pragma unroll
            for (int c = lane; c < CPR; c += 32) {
                const int64_t x = x0 - R + c * VEC;
                float *d = s_tile + r * STRIDE + c * VEC;
                if (x >= 0 && x < nx) {
                    stage16<S>(d, src + c * VEC);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; q += 4) *reinterpret_cast<float4 *>(d + q) = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            }
        }
        cp_async_wait_all();
    } else {
        for (int e = tid; e < kConTR * W; e += kConThreads) {
            const int r = e / W, c = e % W;
            const int64_t row = r0 + r, x = x0 - R + c;
            float v = 0.0f;
            if (row < rows && x >= 0 && x < nx) v = FieldIO<S>::load(in + row * nx + x);
            s_tile[r * STRIDE + c] = v;
        }
    }
    __syncthreads();

    float acc[kConM];
#pragma unroll
    for (int i = 0; i < kConM; i++) acc[i] = 0.0f;
    const float *s = s_tile + lane * STRIDE + warp * kConM;
#pragma unroll
    for (int j4 = 0; j4 < NJ; j4 += 4) {
        const float4 q = *reinterpret_cast<const float4 *>(s + j4);
        const float vv[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int j = j4 + u;
#pragma unroll
            for (int i = 0; i < kConM; i++) {
                const int t = j - i;
                if (t >= 0 && t <= 2 * R) acc[i] = fmaf(taps.k[t], vv[u], acc[i]);
            }
        }
    }
    if (EF && !FINAL) {
        const int64_t row = r0 + lane, xs = x0 + warp * kConM;
        if (row < rows && xs < nx) {
            const int count = nx - xs < kConM ? (int) (nx - xs) : kConM;
            const uint32_t m = mask32<MASK_FMT>(mask, row * nx + xs, count, rows * nx);
            float carry = 0.0f;
#pragma unroll
            for (int i = 0; i < kConM; i++) {
                if ((m >> i) & 1u) {
                    acc[i] = 1.0f;
                    carry = 0.0f;
                } else {
                    const float w = acc[i] + carry;
                    const float q = FieldIO<S>::widen(FieldIO<S>::narrow(w));
                    carry = w - q;
                    acc[i] = q;
                }
            }
        }
    }
    __syncthreads();
    float *so = s_tile + lane * STRIDE + warp * kConM;
#pragma unroll
    for (int i = 0; i < kConM; i += 4)
        *reinterpret_cast<float4 *>(so + i) = make_float4(acc[i], acc[i + 1], acc[i + 2], acc[i + 3]);
    __syncthreads();

    if (vec) {
        // Vector epilogue: 4 voxels per lane-chunk (nx % 4 == 0, so a chunk is
        // either inside the row or past its end).
#pragma unroll
        for (int rr = 0; rr < kConTR / kConWarps; rr++) {
            const int r = warp + rr * kConWarps;
            const int64_t rowbase = (r0 + r) * nx + x0;
#pragma unroll
            for (int c = lane * 4; c < kConTX; c += 128) {
                if (x0 + c >= nx) continue;
                const float4 q = *reinterpret_cast<const float4 *>(s_tile + r * STRIDE + c);
                const int64_t idx = rowbase + c;
                const uint32_t m = mask4<MASK_FMT>(mask, idx);
                const float v0 = (m & 1u) ? 1.0f : q.x, v1 = (m & 2u) ? 1.0f : q.y;
                const float v2 = (m & 4u) ? 1.0f : q.z, v3 = (m & 8u) ? 1.0f : q.w;
                if (FINAL) {
                    if (out_u16) {
                        ushort4 u;
                        u.x = quantise_u16(v0); u.y = quantise_u16(v1);
                        u.z = quantise_u16(v2); u.w = quantise_u16(v3);
                        *reinterpret_cast<ushort4 *>(out_u16 + idx) = u;
                    }
                    if (field_out) *reinterpret_cast<float4 *>(field_out + idx) = make_float4(v0, v1, v2, v3);
                } else {
                    store4<S>(out + idx, v0, v1, v2, v3);
                }
            }
        }
        return;
    }
    for (int e = tid; e < kConTR * kConTX; e += kConThreads) {
        const int r = e / kConTX, c = e % kConTX;
        const int64_t row = r0 + r, x = x0 + c;
        if (row >= rows || x >= nx) continue;
        const int64_t idx = row * nx + x;
        float v = s_tile[r * STRIDE + c];
        if (MaskIO<MASK_FMT>::get(mask, idx)) v = 1.0f;  // re-illumination
        if (FINAL) {
            if (out_u16) out_u16[idx] = quantise_u16(v);
            if (field_out) field_out[idx] = v;
        } else {
            out[idx] = FieldIO<S>::narrow(v);
        }
    }
}

// ---- generic pass (any radius, FP64, reference rounding) -------------------
// One output per thread, direct reads along the axis.  Used for the FP64
// error-reference form, for bit-identical reference rounding (separate
// multiply and add, tap range clipped as in diffusion.cc:41-54) and for radii
// above kMaxUnrolledRadius.
template <typename Acc> struct GenericTaps { Acc k[2 * kMaxRadius + 1]; };

// Rounded multiply and add that the compiler may not fuse into an FMA.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }

template <typename S, bool EXACT, bool X_PASS, int MASK_FMT, bool FINAL>
__global__ void __launch_bounds__(256)
generic_pass(const S *__restrict__ in, S *__restrict__ out, const void *__restrict__ mask,
             uint16_t *__restrict__ out_u16, void *__restrict__ field_out,
             int64_t n, int64_t A, int64_t stride, int radius,
             const GenericTaps<typename FieldIO<S>::Acc> taps) {
    using Acc = typename FieldIO<S>::Acc;
    const int64_t idx = (int64_t) blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const int64_t a = (idx / stride) % A;
    const int64_t lo = -(a < radius ? a : (int64_t) radius);
    const int64_t hi = (A - a - 1 < radius) ? A - a - 1 : (int64_t) radius;
    Acc sum = Acc(0);
    for (int64_t t = lo; t <= hi; t++) {
        const Acc v = FieldIO<S>::load(in + idx + t * stride);
        if (EXACT) sum = add_rn(sum, mul_rn(v, taps.k[radius + t]));
        else sum = fma(taps.k[radius + t], v, sum);
    }
    if (X_PASS) {
        if (MaskIO<MASK_FMT>::get(mask, idx)) sum = Acc(1);
        if (FINAL) {
            if (out_u16) out_u16[idx] = quantise_u16(sum);
            if (field_out) static_cast<Acc *>(field_out)[idx] = sum;
            return;
        }
    }
    out[idx] = FieldIO<S>::narrow(sum);
}

// Rebuilds the bit-packed mask as `field == 1` (the reference's store_mask,
// src/lib/cpp/cpu/diffusion.cc:304-312, used by its on-disk variant).
template <typename S>
__global__ void mask_from_field(const S *__restrict__ field, uint32_t *__restrict__ packed, int64_t n) {
    const int64_t words = (n + 31) / 32;
    for (int64_t w = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (int64_t) gridDim.x * blockDim.x) {
        uint32_t bits = 0;
        for (int j = 0; j < 32; j++) {
            const int64_t i = w * 32 + j;
            if (i < n && FieldIO<S>::widen(field[i]) == 1.0f) bits |= 1u << (31 - j);
        }
        packed[w] = bits;
    }
}

// mask -> {0, 1} field (src/lib/cpp/cpu/diffusion.cc:243-247); with FINAL set
// (zero repetitions) the quantised output and field are written directly.
template <typename S, int MASK_FMT, bool FINAL>
__global__ void mask_to_field(const void *__restrict__ mask, S *__restrict__ field,
                              uint16_t *__restrict__ out_u16, void *__restrict__ field_out, int64_t n) {
    using Acc = typename FieldIO<S>::Acc;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t) gridDim.x * blockDim.x) {
        const bool m = MaskIO<MASK_FMT>::get(mask, i);
        if (FINAL) {
            if (out_u16) out_u16[i] = m ? 65535 : 0;
            if (field_out) static_cast<Acc *>(field_out)[i] = m ? Acc(1) : Acc(0);
        } else {
            field[i] = FieldIO<S>::narrow(m ? Acc(1) : Acc(0));
        }
    }
}

// FP32 field -> storage type (the start of an out-of-core exchange round, which
// continues from the field of the previous round; `src` may be mapped host memory).
template <typename S>
__global__ void field_from_f32(const float *__restrict__ src, S *__restrict__ field, int64_t n) {
    using Acc = typename FieldIO<S>::Acc;
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x)
        field[i] = FieldIO<S>::narrow((Acc) src[i]);
}

}  // namespace maxi
