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
