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

namespace maxi {
namespace tc {

constexpr int kTM = 128;      // outputs along the axis per tile
constexpr int kTN = 128;      // x columns per tile
constexpr int kStages = 2;    // TMA ring depth
constexpr int kThreads = 192; // 6 warps

struct StridedParams {
    void *out;
    int64_t A;          // axis length
    int64_t n_other;    // the third coordinate (y for the z pass, z for the y pass)
    int64_t nx;
    int64_t stride_a;   // element stride along the axis in `out`
    int64_t stride_o;   // element stride of the third coordinate
    int n_at, n_xc;     // axis tiles, x chunks
    int64_t n_tiles;
    int radius, kp, kpa; // radius, K (multiple of 16), K rounded to 64
    int axis_is_z;
    float inv_scale;
    int error_feedback;
    uint16_t hi[2 * kTcMaxRadius + 1];
    uint16_t lo[2 * kTcMaxRadius + 1];
};

__host__ __device__ constexpr int strided_smem_bytes(int kp, int kpa) {
    return 1024 /*alignment slack*/ + 2 * kpa * kTM * 2 /*T_hi, T_lo*/ + kStages * (kTN / 64) * kp * 128 /*B ring*/ +
           256 /*barriers, TMEM slot*/;
}

template <typename S> struct Narrow16;
template <> struct Narrow16<__nv_bfloat16> {
    static __device__ __forceinline__ uint16_t bits(float v, float &carry, bool ef) {
        const float w = ef ? v + carry : v;
        const __nv_bfloat16 q = __float2bfloat16_rn(w);
        if (ef) carry = w - __bfloat162float(q);
        return __bfloat16_as_ushort(q);
    }
};
template <> struct Narrow16<__half> {
    static __device__ __forceinline__ uint16_t bits(float v, float &carry, bool ef) {
        const float w = ef ? v + carry : v;
        const __half q = __float2half_rn(w);
        if (ef) carry = w - __half2float(q);
        return __half_as_ushort(q);
    }
};

template <typename S>
__global__ void __launch_bounds__(kThreads, 1)
tc_strided_pass(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ StridedParams p) {
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
        for (int s = 0; s < kStages; s++) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int d = 0; d < 2; d++) { mbar_init(&tfull[d], 1); mbar_init(&tempty[d], 4); }
        fence_barrier_init();
        prefetch_tmap(&tmap);
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
        // TMA producer.
        int64_t tl = 0;
        for (int64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x, tl++) {
            const int s = (int) (tl % kStages);
            const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
            if (!mbar_wait(&empty[s], ph ^ 1, 1)) break;
            const int at = (int) (tile % p.n_at);
            const int64_t rest = tile / p.n_at;
            const int xc = (int) (rest % p.n_xc);
            const int oth = (int) (rest / p.n_xc);
            const int a_in = at * kTM - p.radius;
            const int x0 = xc * kTN;
            mbar_arrive_expect_tx(&full[s], stage_bytes);
            for (int c = 0; c < kTN / 64; c++) {
                uint8_t *dst = ring + s * stage_bytes + c * p.kp * 128;
                if (p.axis_is_z) tma_load_3d(dst, &tmap, x0 + 64 * c, oth, a_in, &full[s]);
                else tma_load_3d(dst, &tmap, x0 + 64 * c, a_in, oth, &full[s]);
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer.
        const uint32_t fmt = std::is_same<S, __nv_bfloat16>::value ? 1u : 0u;
        const uint32_t idesc = idesc_f16(fmt, 0 /*A K-major*/, 1 /*B MN-major*/, kTM, kTN);
        const uint32_t a_hi = smem_u32(t_hi), a_lo = smem_u32(t_lo), b0 = smem_u32(ring);
        int64_t tl = 0;
        for (int64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x, tl++) {
            const int s = (int) (tl % kStages);
            const uint32_t ph = (uint32_t) ((tl / kStages) & 1);
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&full[s], ph, 1)) break;
            if (!mbar_wait(&tempty[d], dph ^ 1, 3)) break;
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
    } else if (warp >= 2) {
        // Epilogue: TMEM -> registers -> storage type -> global.
        const int quad = warp & 3;           // TMEM lane quadrant this warp may access
        const int o = quad * 32 + lane;      // output row within the tile
        S *out = static_cast<S *>(p.out);
        int64_t tl = 0;
        for (int64_t tile = blockIdx.x; tile < p.n_tiles; tile += gridDim.x, tl++) {
            const int d = (int) (tl & 1);
            const uint32_t dph = (uint32_t) ((tl >> 1) & 1);
            if (!mbar_wait(&tfull[d], dph, 2)) break;
            tc_fence_after();
            const int at = (int) (tile % p.n_at);
            const int64_t rest = tile / p.n_at;
            const int xc = (int) (rest % p.n_xc);
            const int64_t oth = rest / p.n_xc;
            const int64_t a = (int64_t) at * kTM + o;
            const int64_t x0 = (int64_t) xc * kTN;
            float carry = 0.0f;
#pragma unroll 1
            for (int c = 0; c < kTN / 32; c++) {
                float v[32];
                __syncwarp();
                tmem_ld32(tmem + ((uint32_t) (quad * 32) << 16) + d * kTN + c * 32, v);
                if (a >= p.A) continue;
                const int64_t xb = x0 + c * 32;
                S *dst = out + a * p.stride_a + oth * p.stride_o + xb;
                uint16_t q[32];
#pragma unroll
                for (int i = 0; i < 32; i++) q[i] = Narrow16<S>::bits(v[i] * p.inv_scale, carry, p.error_feedback);
                if (xb + 32 <= p.nx) {
#pragma unroll
                    for (int i = 0; i < 32; i += 8) {
                        uint4 u;
                        u.x = q[i] | ((uint32_t) q[i + 1] << 16);
                        u.y = q[i + 2] | ((uint32_t) q[i + 3] << 16);
                        u.z = q[i + 4] | ((uint32_t) q[i + 5] << 16);
                        u.w = q[i + 6] | ((uint32_t) q[i + 7] << 16);
                        *reinterpret_cast<uint4 *>(dst + i) = u;
                    }
                } else {
                    for (int i = 0; i < 32 && xb + i < p.nx; i++) reinterpret_cast<uint16_t *>(dst)[i] = q[i];
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
        tmem_dealloc(tmem, 2 * kTN);
    }
}

// ---- host side -----------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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
    return major == 10 && encode_fn() != nullptr;
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
    for (int i = 0; i < 2 * radius + 1; i++) {
        const float k = kernel[i] * scale;
        if (is_bf16) {
            p.hi[i] = bits_bf16(k);
            p.lo[i] = bits_bf16(k - from_bf16(p.hi[i]));
        } else {
            p.hi[i] = bits_f16(k);
            p.lo[i] = bits_f16(k - from_f16(p.hi[i]));
        }
    }
    if (axis_z) { p.A = nz; p.n_other = ny; p.stride_a = ny * nx; p.stride_o = nx; }
    else { p.A = ny; p.n_other = nz; p.stride_a = nx; p.stride_o = ny * nx; }
    p.n_at = (int) ceil_div(p.A, kTM);
    p.n_xc = (int) ceil_div(nx, kTN);
    p.n_tiles = (int64_t) p.n_at * p.n_xc * p.n_other;

    CUtensorMap map;
    const cuuint64_t dims[3] = {(cuuint64_t) nx, (cuuint64_t) ny, (cuuint64_t) nz};
    const cuuint64_t strides[2] = {(cuuint64_t) (nx * 2), (cuuint64_t) (nx * ny * 2)};
    const cuuint32_t box[3] = {64u, axis_z ? 1u : (cuuint32_t) p.kp, axis_z ? (cuuint32_t) p.kp : 1u};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult cr = encode_fn()(&map, is_bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 3,
                              const_cast<S *>(in), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                              CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (cr != CUDA_SUCCESS) return cudaErrorInvalidValue;

    const int smem = strided_smem_bytes(p.kp, p.kpa);
    cudaError_t e = cudaFuncSetAttribute(tc_strided_pass<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t grid = std::min<int64_t>(p.n_tiles, sms);
    tc_strided_pass<S><<<(unsigned) grid, kThreads, smem, st>>>(map, p);
    return cudaGetLastError();
}

template cudaError_t tc_strided<__nv_bfloat16>(const __nv_bfloat16 *, __nv_bfloat16 *, int64_t, int64_t, int64_t,
                                               bool, const float *, int, bool, cudaStream_t);
template cudaError_t tc_strided<__half>(const __half *, __half *, int64_t, int64_t, int64_t, bool, const float *, int,
                                        bool, cudaStream_t);

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
