// Unrolled CUDA-core repetition loop (template definitions); included by the
// per-type instantiation units passes_f32.cu, passes_bf16.cu, passes_f16.cu.
#pragma once

#include "passes.cuh"
#include "unrolled.h"
#include "profiler.h"
#include "tc_pass.h"

namespace maxi {

// Radii with an unrolled instantiation; a radius between two of these runs
// with the next larger one and zero-padded taps (FMAs with a zero coefficient
// leave the FP32 sum unchanged).
static const int kRadiusBuckets[] = {1, 2, 3, 4, 6, 8, 12, 16, 24, 32, 48, 64, 96, 128};

inline int radius_bucket_impl(int r) {
    for (int b : kRadiusBuckets)
        if (r <= b) return b;
    return -1;
}

template <int R>
static Taps<R> make_taps(const float *kernel, int radius) {
    Taps<R> t;
    for (int i = 0; i < 2 * R + 1; i++) {
        const int off = i - R;
        t.k[i] = (off >= -radius && off <= radius) ? kernel[radius + off] : 0.0f;
    }
    return t;
}

template <typename F>
static cudaError_t set_smem(F *f, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

// One repetition loop for bucket radius R.  EF: error-feedback rounding of the
// 16-bit storage type (see passes.cuh); use_tc: z and y passes on the tensor
// cores (16-bit storage only, tc_pass.cu).
template <int R, typename S, bool EF>
static cudaError_t run_unrolled(const Volume &v, const void *mask, int mask_fmt, const float *kernel,
                                int radius, int64_t reps, S *buf0, S *buf1, uint16_t *out_u16,
                                float *field_out, bool use_tc, bool fuse_yx, bool hi_only, uint32_t *rebuild_mask,
                                const RunOpts &o, cudaStream_t st) {
    const int64_t shrink_lo = o.shrink_lo, shrink_hi = o.shrink_hi;
    const Taps<R> taps = make_taps<R>(kernel, radius);
    const int str_smem = strided_smem_bytes<R>();
    const int con_smem = contig_smem_bytes<R>();
    auto *zy = strided_pass<R, S, EF>;
    cudaError_t e = set_smem(zy, str_smem);
    if (e != cudaSuccess) return e;
    auto *xu8 = contig_pass<R, S, MAXI_MASK_U8, false, EF>;
    auto *xu8f = contig_pass<R, S, MAXI_MASK_U8, true, EF>;
    auto *xbp = contig_pass<R, S, MAXI_MASK_BITPACKED, false, EF>;
    auto *xbpf = contig_pass<R, S, MAXI_MASK_BITPACKED, true, EF>;
    for (auto *f : {xu8, xu8f, xbp, xbpf})
        if ((e = set_smem(f, con_smem)) != cudaSuccess) return e;
    auto *xpass = mask_fmt == MAXI_MASK_U8 ? xu8 : xbp;
    auto *xfinal = mask_fmt == MAXI_MASK_U8 ? xu8f : xbpf;

    const int64_t n = v.n();
    {
        const int threads = 256;
        const int64_t blocks = std::min<int64_t>((n + threads - 1) / threads, 148 * 64);
        ProfScope ps(MAXI_KERNEL_INIT, st);
        if (o.init_field)
            field_from_f32<S><<<blocks, threads, 0, st>>>(o.init_field, buf0, n);
        else if (mask_fmt == MAXI_MASK_U8)
            mask_to_field<S, MAXI_MASK_U8, false><<<blocks, threads, 0, st>>>(mask, buf0, nullptr, nullptr, n);
        else
            mask_to_field<S, MAXI_MASK_BITPACKED, false><<<blocks, threads, 0, st>>>(mask, buf0, nullptr, nullptr, n);
    }
    const int64_t plane = v.ny * v.nx;
    // Tensor-core x pass: vector epilogue needs 16-byte aligned mask (u8), output and field.
    const bool tc_x = use_tc &&
                      ((reinterpret_cast<uintptr_t>(out_u16) | reinterpret_cast<uintptr_t>(field_out) |
                        (mask_fmt == MAXI_MASK_U8 ? reinterpret_cast<uintptr_t>(mask) : 0)) & 15) == 0;
    // Fused y + x kernel: z pass buf0 -> buf1, y + x buf1 -> buf0 ([y][z][x] rows
    // between repetitions), so the buffers do not swap.
    const bool yx = tc_x && fuse_yx && hi_only && tc::tc_yx_supported(radius, v.nz, v.ny, v.nx);
    if (reps > 0)
        note_path(yx ? (MAXI_PATH_TENSOR_CORES_ZY | MAXI_PATH_FUSED_YX)
                     : ((use_tc ? MAXI_PATH_TENSOR_CORES_ZY : MAXI_PATH_CUDA_CORES) |
                        (tc_x ? MAXI_PATH_TENSOR_CORES_X : MAXI_PATH_CUDA_CORES)));
    for (int64_t rep = 0; rep < reps; rep++) {
        // Plane window of this repetition (the whole volume unless shrinking).
        const int64_t lo = std::min(v.nz - 1, shrink_lo * rep);
        const int64_t hi = std::max(lo + 1, v.nz - shrink_hi * rep);
        const int64_t nzv = hi - lo, off = lo * plane;
        S *b0 = buf0 + off, *b1 = buf1 + off;
        const void *mv = mask_fmt == MAXI_MASK_U8 ? static_cast<const void *>(static_cast<const uint8_t *>(mask) + off)
                                                  : static_cast<const void *>(static_cast<const uint32_t *>(mask) + off / 32);
        uint16_t *ou = out_u16 ? out_u16 + off : nullptr;
        float *fo = field_out ? field_out + off : nullptr;
        // z pass: [1][nzv][ny*nx]; y pass: [nzv][ny][nx]
        const int64_t zI = plane, zA = nzv, zat = ceil_div(zA, kStrTA), zit = ceil_div(zI, kStrTI);
        const int64_t yI = v.nx, yA = v.ny, yO = nzv, yat = ceil_div(yA, kStrTA), yit = ceil_div(yI, kStrTI);
        const int64_t rows = nzv * v.ny, xt = ceil_div(v.nx, kConTX), xrb = ceil_div(rows, kConTR);
        if (o.final_wait && rep + 1 == reps && (e = cudaStreamWaitEvent(st, o.final_wait, 0)) != cudaSuccess) return e;
        // The rebuilt-mask semantics: before every repetition after the first of
        // the whole run (a continued run's first repetition is not the first).
        if (rebuild_mask && (rep > 0 || o.init_field)) {
            ProfScope ps(MAXI_KERNEL_OTHER, st);
            const int64_t blocks = std::min<int64_t>(ceil_div(ceil_div(nzv * plane, 32), 256), 148 * 16);
            mask_from_field<S><<<blocks, 256, 0, st>>>(b0, rebuild_mask + off / 32, nzv * plane);
        }
        {
            ProfScope ps(MAXI_KERNEL_Z, st);
            if constexpr (sizeof(S) == 2) {
                // After the first repetition the tensor-core x pass leaves the field in
                // [y][z][x] row order (over all v.nz planes), which the z pass reads faster.
                const tc::YzRows yz{buf0, v.nz, lo};
                if (use_tc) e = tc::tc_strided<S>(b0, b1, nzv, v.ny, v.nx, true, kernel, radius, EF, st,
                                                  tc_x && rep > 0 ? &yz : nullptr, hi_only);
                else zy<<<zat * zit, kStrThreads, str_smem, st>>>(b0, b1, zA, zI, zat, zit, taps);
            } else {
                zy<<<zat * zit, kStrThreads, str_smem, st>>>(b0, b1, zA, zI, zat, zit, taps);
            }
        }
        if (e != cudaSuccess) return e;
        const bool last = rep + 1 == reps;
        if constexpr (sizeof(S) == 2) {
            if (yx) {
                ProfScope ps(MAXI_KERNEL_YX, st);
                const tc::YzRows yz{buf0, v.nz, lo};
                e = tc::tc_yx<S>(b1, b0, mv, mask_fmt, last, last ? ou : nullptr, last ? fo : nullptr, nzv, v.ny,
                                 v.nx, kernel, radius, EF, hi_only, st, &yz);
                if (e != cudaSuccess) return e;
                continue;
            }
        }
        {
            ProfScope ps(MAXI_KERNEL_Y, st);
            if constexpr (sizeof(S) == 2) {
                if (use_tc) e = tc::tc_strided<S>(b1, b0, nzv, v.ny, v.nx, false, kernel, radius, EF, st, nullptr, hi_only);
                else zy<<<yat * yit * yO, kStrThreads, str_smem, st>>>(b1, b0, yA, yI, yat, yit, taps);
            } else {
                zy<<<yat * yit * yO, kStrThreads, str_smem, st>>>(b1, b0, yA, yI, yat, yit, taps);
            }
        }
        if (e != cudaSuccess) return e;
        {
            ProfScope ps(last ? MAXI_KERNEL_X_FINAL : MAXI_KERNEL_X, st);
            if (tc_x) {
                if constexpr (sizeof(S) == 2) {
                    const tc::YzRows yz{buf1, v.nz, lo};
                    e = tc::tc_contig<S>(b0, b1, mv, mask_fmt, last, last ? ou : nullptr, last ? fo : nullptr, nzv,
                                         v.ny, v.nx, kernel, radius, EF, st, &yz, hi_only);
                }
            } else if (!last) {
                xpass<<<xt * xrb, kConThreads, con_smem, st>>>(b0, b1, mv, nullptr, nullptr, rows, v.nx, xt, taps);
            } else {
                xfinal<<<xt * xrb, kConThreads, con_smem, st>>>(b0, b1, mv, ou, fo, rows, v.nx, xt, taps);
            }
        }
        if (e != cudaSuccess) return e;
        if (!last) std::swap(buf0, buf1);
    }
    return cudaGetLastError();
}

template <typename S>
cudaError_t launch_init_field(const void *mask, int mask_fmt, S *field, int64_t n, cudaStream_t st) {
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), 148 * 64);
    if (mask_fmt == MAXI_MASK_U8)
        mask_to_field<S, MAXI_MASK_U8, false><<<blocks, 256, 0, st>>>(mask, field, nullptr, nullptr, n);
    else
        mask_to_field<S, MAXI_MASK_BITPACKED, false><<<blocks, 256, 0, st>>>(mask, field, nullptr, nullptr, n);
    return cudaGetLastError();
}

template <typename S, bool EF>
static cudaError_t dispatch_radius(const Volume &v, const void *mask, int mask_fmt, const float *kernel, int radius,
                                   int64_t reps, S *b0, S *b1, uint16_t *out_u16, float *field_out, bool use_tc,
                                   bool fuse_yx, bool hi_only, uint32_t *rebuild, const RunOpts &o, cudaStream_t st) {
    switch (radius_bucket_impl(radius)) {
#define MAXI_CASE(RB) \
    case RB: return run_unrolled<RB, S, EF>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16, field_out, use_tc, fuse_yx, hi_only, rebuild, o, st);
        MAXI_CASE(1) MAXI_CASE(2) MAXI_CASE(3) MAXI_CASE(4) MAXI_CASE(6) MAXI_CASE(8) MAXI_CASE(12)
        MAXI_CASE(16) MAXI_CASE(24) MAXI_CASE(32) MAXI_CASE(48) MAXI_CASE(64) MAXI_CASE(96) MAXI_CASE(128)
#undef MAXI_CASE
    default: return cudaErrorInvalidValue;
    }
}

template <typename S>
cudaError_t dispatch_unrolled(const Volume &v, const void *mask, int mask_fmt, const float *kernel, int radius,
                              int64_t reps, S *b0, S *b1, uint16_t *out_u16, float *field_out, int32_t flags,
                              cudaStream_t st, const RunOpts &o) {
    // Mask rebuilt from the field each repetition: the caller passes a writable
    // bit-packed copy (the workspace's).
    uint32_t *rebuild = (flags & MAXI_FLAG_MASK_FROM_FIELD) && mask_fmt == MAXI_MASK_BITPACKED
                            ? const_cast<uint32_t *>(static_cast<const uint32_t *>(mask))
                            : nullptr;
    if constexpr (sizeof(S) == 2) {
        // Error feedback relies on the following x pass to remove high-pass noise;
        // kernels narrower than radius 4 (sigma < 1) pass too much of it.
        const bool ef = (flags & MAXI_FLAG_NEAREST_ROUNDING) == 0 && radius >= 4;
        const bool use_tc = (flags & MAXI_FLAG_NO_TENSOR_CORES) == 0 && tc::tc_supported(radius, v.nz, v.ny, v.nx);
        // The rebuilt-mask semantics rewrite the mask between repetitions from the
        // x pass's output; they keep the separate passes.
        const bool fuse = (flags & (MAXI_FLAG_SEPARATE_PASSES | MAXI_FLAG_MASK_FROM_FIELD)) == 0;
        const bool hi_only = tc::tc_single_set(radius, (flags & MAXI_FLAG_SPLIT_COEFFICIENTS) != 0);
        if (ef) return dispatch_radius<S, true>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16, field_out, use_tc, fuse, hi_only, rebuild, o, st);
        return dispatch_radius<S, false>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16, field_out, use_tc, fuse, hi_only, rebuild, o, st);
    } else {
        return dispatch_radius<S, false>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16, field_out, false, false, false, rebuild, o, st);
    }
}

}  // namespace maxi
