// Shared definitions for the mask-diffusion kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include "../../include/maxibone_diffusion.h"

namespace maxi {

// Largest kernel radius served by the unrolled CUDA-core passes; larger radii
// take the generic pass.
constexpr int kMaxUnrolledRadius = 128;
// Largest radius at all (kernel_size <= 2*kMaxRadius+1).
constexpr int kMaxRadius = 1024;

// ---------------------------------------------------------------------------
// Field storage types.  The field lives in HBM as S between passes and is
// widened to the accumulation type on load.
// ---------------------------------------------------------------------------
template <typename S> struct FieldIO;

template <> struct FieldIO<float> {
    using Acc = float;
    static __device__ __forceinline__ float load(const float *p) { return __ldg(p); }
    static __device__ __forceinline__ float widen(float v) { return v; }
    static __device__ __forceinline__ float narrow(float v) { return v; }
};
template <> struct FieldIO<__nv_bfloat16> {
    using Acc = float;
    static __device__ __forceinline__ float load(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
    static __device__ __forceinline__ float widen(__nv_bfloat16 v) { return __bfloat162float(v); }
    static __device__ __forceinline__ __nv_bfloat16 narrow(float v) { return __float2bfloat16_rn(v); }
};
template <> struct FieldIO<__half> {
    using Acc = float;
    static __device__ __forceinline__ float load(const __half *p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ float widen(__half v) { return __half2float(v); }
    static __device__ __forceinline__ __half narrow(float v) { return __float2half_rn(v); }
};
template <> struct FieldIO<double> {
    using Acc = double;
    static __device__ __forceinline__ double load(const double *p) { return __ldg(p); }
    static __device__ __forceinline__ double widen(double v) { return v; }
    static __device__ __forceinline__ double narrow(double v) { return v; }
};

// ---------------------------------------------------------------------------
// 16-byte vector staging: global (aligned) -> shared floats (aligned).
// Float fields use cp.async (no register round trip); 2-byte fields are
// widened in registers (8 values per 16 bytes).
// ---------------------------------------------------------------------------
template <typename S> struct Vec16 { static constexpr int N = 16 / sizeof(S); };

__device__ __forceinline__ void cp_async16(float *smem, const void *gmem) {
    const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <typename S> __device__ __forceinline__ void stage16(float *smem, const S *gmem);
template <> __device__ __forceinline__ void stage16<float>(float *smem, const float *gmem) { cp_async16(smem, gmem); }
template <> __device__ __forceinline__ void stage16<__nv_bfloat16>(float *smem, const __nv_bfloat16 *gmem) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(gmem));
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
    float f[8];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        f[2 * i] = __uint_as_float(w[i] << 16);
        f[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
    }
    reinterpret_cast<float4 *>(smem)[0] = make_float4(f[0], f[1], f[2], f[3]);
    reinterpret_cast<float4 *>(smem)[1] = make_float4(f[4], f[5], f[6], f[7]);
}
template <> __device__ __forceinline__ void stage16<__half>(float *smem, const __half *gmem) {
    const uint4 q = __ldg(reinterpret_cast<const uint4 *>(gmem));
    const __half2 *h = reinterpret_cast<const __half2 *>(&q);
    float f[8];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 t = __half22float2(h[i]);
        f[2 * i] = t.x;
        f[2 * i + 1] = t.y;
    }
    reinterpret_cast<float4 *>(smem)[0] = make_float4(f[0], f[1], f[2], f[3]);
    reinterpret_cast<float4 *>(smem)[1] = make_float4(f[4], f[5], f[6], f[7]);
}

// Stores 4 consecutive values (destination aligned to 4 elements).
template <typename S> __device__ __forceinline__ void store4(S *dst, float a, float b, float c, float d);
template <> __device__ __forceinline__ void store4<float>(float *dst, float a, float b, float c, float d) {
    *reinterpret_cast<float4 *>(dst) = make_float4(a, b, c, d);
}
template <> __device__ __forceinline__ void store4<__nv_bfloat16>(__nv_bfloat16 *dst, float a, float b, float c, float d) {
    const __nv_bfloat162 lo = __floats2bfloat162_rn(a, b), hi = __floats2bfloat162_rn(c, d);
    uint2 u;
    u.x = *reinterpret_cast<const uint32_t *>(&lo);
    u.y = *reinterpret_cast<const uint32_t *>(&hi);
    *reinterpret_cast<uint2 *>(dst) = u;
}
template <> __device__ __forceinline__ void store4<__half>(__half *dst, float a, float b, float c, float d) {
    const __half2 lo = __floats2half2_rn(a, b), hi = __floats2half2_rn(c, d);
    uint2 u;
    u.x = *reinterpret_cast<const uint32_t *>(&lo);
    u.y = *reinterpret_cast<const uint32_t *>(&hi);
    *reinterpret_cast<uint2 *>(dst) = u;
}

// ---------------------------------------------------------------------------
// Mask access.  U8: set when the byte is > 0 (the reference's `mask > 0`).
// Bit-packed: flat voxel order, uint32 words, most significant bit first.
// ---------------------------------------------------------------------------
template <int FMT> struct MaskIO;
template <> struct MaskIO<MAXI_MASK_U8> {
    static __device__ __forceinline__ bool get(const void *m, int64_t i) {
        return __ldg(static_cast<const uint8_t *>(m) + i) > 0;
    }
};
template <> struct MaskIO<MAXI_MASK_BITPACKED> {
    static __device__ __forceinline__ bool get(const void *m, int64_t i) {
        const uint32_t w = __ldg(static_cast<const uint32_t *>(m) + (i >> 5));
        return (w >> (31 - (int) (i & 31))) & 1u;
    }
};

// Four consecutive mask flags starting at a voxel index that is a multiple of 4
// (bit q of the result = voxel i + q).
template <int FMT> __device__ __forceinline__ uint32_t mask4(const void *m, int64_t i);
template <> __device__ __forceinline__ uint32_t mask4<MAXI_MASK_U8>(const void *m, int64_t i) {
    const uint32_t w = __ldg(reinterpret_cast<const uint32_t *>(static_cast<const uint8_t *>(m) + i));
    uint32_t r = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) r |= (((w >> (8 * q)) & 0xffu) != 0u) << q;
    return r;
}
template <> __device__ __forceinline__ uint32_t mask4<MAXI_MASK_BITPACKED>(const void *m, int64_t i) {
    const uint32_t w = __ldg(static_cast<const uint32_t *>(m) + (i >> 5));
    const uint32_t nib = (w >> (28 - (int) (i & 31))) & 0xfu;  // bits for voxels i..i+3, MSB first
    return __brev(nib) >> 28;                                   // reorder: bit q = voxel i + q
}

// Mask flags of up to 32 consecutive voxels [i, i + count) of a row (bit q =
// voxel i + q; bits at or above `count` are zero).  `n` is the volume size,
// bounding the bit-packed words read.
template <int FMT> __device__ __forceinline__ uint32_t mask32(const void *m, int64_t i, int count, int64_t n);
template <> __device__ __forceinline__ uint32_t mask32<MAXI_MASK_U8>(const void *m, int64_t i, int count, int64_t n) {
    const uint8_t *p = static_cast<const uint8_t *>(m) + i;
    uint32_t r = 0;
    for (int q = 0; q < count; q++) r |= (uint32_t) (__ldg(p + q) != 0) << q;
    return r;
}
template <> __device__ __forceinline__ uint32_t mask32<MAXI_MASK_BITPACKED>(const void *m, int64_t i, int count, int64_t n) {
    const uint32_t *w = static_cast<const uint32_t *>(m);
    const int64_t w0 = i >> 5;
    const int b = (int) (i & 31);
    const uint64_t hi = __ldg(w + w0);
    const uint64_t lo = (b > 0 && (w0 + 1) * 32 < n) ? __ldg(w + w0 + 1) : 0u;
    const uint32_t msb_first = (uint32_t) ((((hi << 32) | lo) << b) >> 32);  // voxel i at bit 31
    const uint32_t r = __brev(msb_first);                                      // voxel i at bit 0
    return count >= 32 ? r : (r & ((1u << count) - 1u));
}

// Quantisation of the reference (src/lib/cpp/cpu/diffusion.cc:191-195):
// floor(v * 65535.0f) in FP32, clamped to the uint16 range.
__device__ __forceinline__ uint16_t quantise_u16(float v) {
    float q = floorf(v * 65535.0f);
    q = fminf(fmaxf(q, 0.0f), 65535.0f);
    return (uint16_t) q;
}
__device__ __forceinline__ uint16_t quantise_u16(double v) {
    double q = floor(v * 65535.0);
    q = fmin(fmax(q, 0.0), 65535.0);
    return (uint16_t) q;
}

}  // namespace maxi
