// sm_100a primitives for the tensor-core passes: mbarriers with bounded waits,
// TMA tile loads, tcgen05 (TMEM allocation, UMMA, commit, loads), and the
// shared-memory matrix / instruction descriptors of tcgen05.mma kind::f16.
//
// Every wait on an mbarrier is bounded by a clock budget (about one second at
// the B200 clock); on timeout the waiting thread records an error code in
// the device error word and returns false, so a kernel never spins forever.
#pragma once

#include <cuda.h>
#include <stdint.h>

#include "common.cuh"

namespace maxi {
namespace tc {

// Device error word of the tensor-core passes (0 = fine).  Codes: 1 = a TMA
// tile never arrived, 2 = MMAs never completed, 3 = the accumulator was never
// released by the epilogue.
static __device__ int g_tc_error = 0;

constexpr long long kWaitBudgetCycles = 2000000000ll;  // ~1 s at 1.9 GHz

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.shared::cta.b64 st, [%0];\n}\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n}\n"
                 ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
    return ok != 0;
}

// As mbar_try_wait, letting the hardware suspend the thread until the phase
// completes or `suspend_ns` nanoseconds pass, instead of returning at once: a
// waiting warp then takes no issue slots from the warps doing the work.
__device__ __forceinline__ bool mbar_try_wait_suspend(uint64_t *bar, uint32_t parity, uint32_t suspend_ns) {
    uint32_t ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity), "r"(suspend_ns) : "memory");
    return ok != 0;
}

constexpr uint32_t kWaitSuspendNs = 1000000;  // per try: 1 ms, far inside the bounded wait's ~1 s

// Bounded wait for the phase with the given parity to complete.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int err_code) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait_suspend(bar, parity, kWaitSuspendNs)) {
        if (clock64() - t0 > kWaitBudgetCycles) {
            atomicCAS(&g_tc_error, 0, err_code);
            return false;
        }
    }
    return true;
}

// 3-D tiled TMA load into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_3d(void *smem, const CUtensorMap *map, int c0, int c1, int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];\n"
        ::"r"(smem_u32(smem)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
        : "memory");
}

// Prefetch of a 3-D tile into L2 (no shared-memory destination).
__device__ __forceinline__ void tma_prefetch_3d(const CUtensorMap *map, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.prefetch.tensor.3d.L2.global [%0, {%1, %2, %3}];\n"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2) : "memory");
}

// 3-D tiled TMA store from shared memory (bulk async-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap *map, const void *smem, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];\n"
                 ::"l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(smem)), "r"(c0), "r"(c1), "r"(c2) : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// Waits until at most N committed bulk groups still read their shared-memory source.
template <int N> __device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap *map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// ---- TMEM ------------------------------------------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// D[tmem] (+)= A[smem desc] * B[smem desc]; issued by one thread.
__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n"
        ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate) : "memory");
}

// As umma_f16 with the A operand in tensor memory (K-major: row m in lane m,
// two 16-bit K elements per 32-bit column).
__device__ __forceinline__ void umma_f16_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n}\n"
        ::"r"(d_tmem), "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate) : "memory");
}

// Arrives on `bar` once all previously issued tcgen05.mma of this thread complete.
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n"
                 ::"r"(smem_u32(bar)) : "memory");
}

// 32 lanes x 32 columns of 32-bit: thread (lane) l of the warp gets columns
// [col, col+32) of TMEM lane (quadrant base + l).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; i++) v[i] = __uint_as_float(r[i]);
}

// As tmem_ld32 for 64 columns [col, col+64) in one load.
__device__ __forceinline__ void tmem_ld64(uint32_t taddr, float (&v)[64]) {
    uint32_t r[64];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x64.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, "
        "%32, %33, %34, %35, %36, %37, %38, %39, %40, %41, %42, %43, %44, %45, %46, %47, "
        "%48, %49, %50, %51, %52, %53, %54, %55, %56, %57, %58, %59, %60, %61, %62, %63}, [%64];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31]),
          "=r"(r[32]), "=r"(r[33]), "=r"(r[34]), "=r"(r[35]), "=r"(r[36]), "=r"(r[37]), "=r"(r[38]), "=r"(r[39]),
          "=r"(r[40]), "=r"(r[41]), "=r"(r[42]), "=r"(r[43]), "=r"(r[44]), "=r"(r[45]), "=r"(r[46]), "=r"(r[47]),
          "=r"(r[48]), "=r"(r[49]), "=r"(r[50]), "=r"(r[51]), "=r"(r[52]), "=r"(r[53]), "=r"(r[54]), "=r"(r[55]),
          "=r"(r[56]), "=r"(r[57]), "=r"(r[58]), "=r"(r[59]), "=r"(r[60]), "=r"(r[61]), "=r"(r[62]), "=r"(r[63])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 64; i++) v[i] = __uint_as_float(r[i]);
}

// Thread (lane) l of the warp writes r[0..31] to columns [col, col+32) of TMEM
// lane (quadrant base + l); tmem_st_wait() waits for the warp's stores.
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&r)[32]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};\n"
        ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
          "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15]),
          "r"(r[16]), "r"(r[17]), "r"(r[18]), "r"(r[19]), "r"(r[20]), "r"(r[21]), "r"(r[22]), "r"(r[23]),
          "r"(r[24]), "r"(r[25]), "r"(r[26]), "r"(r[27]), "r"(r[28]), "r"(r[29]), "r"(r[30]), "r"(r[31])
        : "memory");
}
__device__ __forceinline__ void tmem_st_wait() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }

// Thread (lane) l of the warp writes r[0..15] to columns [col, col+16) of TMEM
// lane (quadrant base + l).
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};\n"
        ::"r"(taddr), "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
          "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
}

// ---- descriptors -------------------------------------------------------------
// Shared-memory matrix descriptor (tcgen05): start address, leading and stride
// byte offsets (16-byte units), version 1, 128-byte swizzle (layout type 2).
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    uint64_t d = 0;
    d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
    d |= (uint64_t) ((lbo_bytes >> 4) & 0x3FFF) << 16;
    d |= (uint64_t) ((sbo_bytes >> 4) & 0x3FFF) << 32;
    d |= (uint64_t) 1 << 46;  // version
    d |= (uint64_t) 2 << 61;  // SWIZZLE_128B
    return d;
}

// Instruction descriptor for kind::f16 with FP32 accumulation.
// fmt: 0 = F16, 1 = BF16; majors: 0 = K-major, 1 = MN-major.
__host__ __device__ constexpr uint32_t idesc_f16(uint32_t fmt, uint32_t a_major, uint32_t b_major, uint32_t m,
                                                 uint32_t n) {
    return (1u << 4) | (fmt << 7) | (fmt << 10) | (a_major << 15) | (b_major << 16) | ((n >> 3) << 17) |
           ((m >> 4) << 24);
}

// Byte offset of element (row, k) of a K-major, 128-byte-swizzled operand with
// 64-element K blocks of `rows` rows each (16-bit elements).
__device__ __forceinline__ uint32_t sw128_kmajor_offset(int row, int k, int rows) {
    const int kb = k >> 6, kin = k & 63;
    const int chunk = kin >> 3, within = (kin & 7) * 2;
    return kb * rows * 128 + (row >> 3) * 1024 + (row & 7) * 128 + ((chunk ^ (row & 7)) << 4) + within;
}

// Rounds to the 16-bit storage type; with `ef` the rounding error is carried
// into the next value of the chain (error feedback).
template <typename S> struct Narrow16;
template <> struct Narrow16<__nv_bfloat16> {
    static __device__ __forceinline__ uint16_t bits(float v, float &carry, bool ef) {
        const float w = ef ? v + carry : v;
        const __nv_bfloat16 q = __float2bfloat16_rn(w);
        if (ef) carry = w - __bfloat162float(q);
        return __bfloat16_as_ushort(q);
    }
    static __device__ __forceinline__ float widen(uint16_t q) { return __uint_as_float((uint32_t) q << 16); }
};
template <> struct Narrow16<__half> {
    static __device__ __forceinline__ uint16_t bits(float v, float &carry, bool ef) {
        const float w = ef ? v + carry : v;
        const __half q = __float2half_rn(w);
        if (ef) carry = w - __half2float(q);
        return __half_as_ushort(q);
    }
    static __device__ __forceinline__ float widen(uint16_t q) { return __half2float(__ushort_as_half(q)); }
};

// Narrows one 32-voxel chunk (32 consecutive x voxels) to the 16-bit storage
// type.  With `ef`, rounding errors are carried along x in two interleaved
// chains of 16 voxels (independent carries give the scheduler two instruction
// streams instead of one serial chain).  Voxels whose mask bit is set are
// stored as exactly 1.0; 1.0 is exact in both storage types, so such a voxel
// also hands a zero carry to its neighbour.  `scale` undoes the coefficient
// scaling of the MMA.
template <typename S>
__device__ __forceinline__ void narrow32_masked(const float (&a)[32], uint32_t ma, float scale, bool ef,
                                                uint16_t (&qa)[32]) {
    float c[2] = {0.0f, 0.0f};
#pragma unroll
    for (int j = 0; j < 16; j++) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int i = k * 16 + j;
            const bool mk = (ma >> i) & 1u;
            const float w = mk ? 1.0f : (ef ? fmaf(a[i], scale, c[k]) : a[i] * scale);
            float dummy = 0.0f;
            const uint16_t q = Narrow16<S>::bits(w, dummy, false);
            if (ef) c[k] = w - Narrow16<S>::widen(q);
            qa[i] = q;
        }
    }
}

// One 32-voxel chunk, no mask: two interleaved 16-voxel error-feedback chains.
template <typename S>
__device__ __forceinline__ void narrow32(const float (&a)[32], float scale, bool ef, uint16_t (&qa)[32]) {
    float c[2] = {0.0f, 0.0f};
#pragma unroll
    for (int j = 0; j < 16; j++) {
#pragma unroll
        for (int k = 0; k < 2; k++) {
            const int i = k * 16 + j;
            const float w = ef ? fmaf(a[i], scale, c[k]) : a[i] * scale;
            float dummy = 0.0f;
            const uint16_t q = Narrow16<S>::bits(w, dummy, false);
            if (ef) c[k] = w - Narrow16<S>::widen(q);
            qa[i] = q;
        }
    }
}

// Two 16-bit values from one paired conversion (low half: the first value)
// and back to FP32.
template <typename S> struct Pair16;
template <> struct Pair16<__nv_bfloat16> {
    static __device__ __forceinline__ uint32_t cvt(float lo, float hi) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
    static __device__ __forceinline__ float2 widen(uint32_t q) {
        return make_float2(__uint_as_float(q << 16), __uint_as_float(q & 0xffff0000u));
    }
};
template <> struct Pair16<__half> {
    static __device__ __forceinline__ uint32_t cvt(float lo, float hi) {
        const __half2 h = __floats2half2_rn(lo, hi);
        return *reinterpret_cast<const uint32_t *>(&h);
    }
    static __device__ __forceinline__ float2 widen(uint32_t q) {
        return __half22float2(*reinterpret_cast<const __half2 *>(&q));
    }
};

// One 32-voxel chunk narrowed to the storage type two voxels per instruction:
// the two error-feedback chains (x = j and x = 16 + j, j = 0..15) advance
// together -- w = a * scale + carry as one packed FMA, one paired conversion,
// the carries w - q as one packed FMA -- which is the per-voxel arithmetic of
// narrow32 / narrow32_masked (bit for bit), in about half the instructions.
// MASKED: voxels with their bit set in `force1` store exactly 1.0
// (re-illumination), voxels with their bit clear in `live` store exactly 0
// (outside the volume); both hand a zero carry on.  d[j] holds voxels j (low
// half) and 16 + j (high half).
template <typename S, bool MASKED>
__device__ __forceinline__ void narrow32_pairs(const float (&a)[32], float scale, bool ef, uint32_t force1,
                                               uint32_t live, uint32_t (&d)[16]) {
    float2 c = make_float2(0.0f, 0.0f);
    const float2 s2 = make_float2(scale, scale), m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const float2 v = make_float2(a[j], a[16 + j]);
        float2 w = ef ? __ffma2_rn(v, s2, c) : __fmul2_rn(v, s2);
        if (MASKED) {
            if (!((live >> j) & 1u)) w.x = 0.0f;
            if (!((live >> (16 + j)) & 1u)) w.y = 0.0f;
            if ((force1 >> j) & 1u) w.x = 1.0f;
            if ((force1 >> (16 + j)) & 1u) w.y = 1.0f;
        }
        const uint32_t q = Pair16<S>::cvt(w.x, w.y);
        if (ef) c = __ffma2_rn(Pair16<S>::widen(q), m1, w);
        d[j] = q;
    }
}

// Two 32-voxel runs narrowed together, each exactly as narrow32_pairs<S, true>
// with live = all and its own force1 (f0: a[0..31] -> d0, f1: a[32..63] -> d1):
// the runs' chains are independent, so every step issues both.
template <typename S>
__device__ __forceinline__ void narrow64_pairs_forced(const float (&a)[64], float scale, bool ef, uint32_t f0,
                                                      uint32_t f1, uint32_t (&d0)[16], uint32_t (&d1)[16]) {
    float2 c0 = make_float2(0.0f, 0.0f), c1 = make_float2(0.0f, 0.0f);
    const float2 s2 = make_float2(scale, scale), m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const float2 v0 = make_float2(a[j], a[16 + j]), v1 = make_float2(a[32 + j], a[48 + j]);
        float2 w0 = ef ? __ffma2_rn(v0, s2, c0) : __fmul2_rn(v0, s2);
        float2 w1 = ef ? __ffma2_rn(v1, s2, c1) : __fmul2_rn(v1, s2);
        if ((f0 >> j) & 1u) w0.x = 1.0f;
        if ((f0 >> (16 + j)) & 1u) w0.y = 1.0f;
        if ((f1 >> j) & 1u) w1.x = 1.0f;
        if ((f1 >> (16 + j)) & 1u) w1.y = 1.0f;
        const uint32_t q0 = Pair16<S>::cvt(w0.x, w0.y), q1 = Pair16<S>::cvt(w1.x, w1.y);
        if (ef) {
            c0 = __ffma2_rn(Pair16<S>::widen(q0), m1, w0);
            c1 = __ffma2_rn(Pair16<S>::widen(q1), m1, w1);
        }
        d0[j] = q0;
        d1[j] = q1;
    }
}

// narrow64_pairs_forced with the voxels of each step in adjacent elements:
// a[2j], a[2j + 1] are voxels j and 16 + j of the first run, a[32 + 2j],
// a[33 + 2j] those of the second (a permuted tensor-memory column order).
// Bit for bit the same rounding as narrow64_pairs_forced.
template <typename S>
__device__ __forceinline__ void narrow64_pairs_forced_adjacent(const float (&a)[64], float scale, bool ef, uint32_t f0,
                                                               uint32_t f1, uint32_t (&d0)[16], uint32_t (&d1)[16]) {
    float2 c0 = make_float2(0.0f, 0.0f), c1 = make_float2(0.0f, 0.0f);
    const float2 s2 = make_float2(scale, scale), m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
    for (int j = 0; j < 16; j++) {
        const float2 v0 = make_float2(a[2 * j], a[2 * j + 1]), v1 = make_float2(a[32 + 2 * j], a[33 + 2 * j]);
        float2 w0 = ef ? __ffma2_rn(v0, s2, c0) : __fmul2_rn(v0, s2);
        float2 w1 = ef ? __ffma2_rn(v1, s2, c1) : __fmul2_rn(v1, s2);
        if ((f0 >> j) & 1u) w0.x = 1.0f;
        if ((f0 >> (16 + j)) & 1u) w0.y = 1.0f;
        if ((f1 >> j) & 1u) w1.x = 1.0f;
        if ((f1 >> (16 + j)) & 1u) w1.y = 1.0f;
        const uint32_t q0 = Pair16<S>::cvt(w0.x, w0.y), q1 = Pair16<S>::cvt(w1.x, w1.y);
        if (ef) {
            c0 = __ffma2_rn(Pair16<S>::widen(q0), m1, w0);
            c1 = __ffma2_rn(Pair16<S>::widen(q1), m1, w1);
        }
        d0[j] = q0;
        d1[j] = q1;
    }
}

// 32 voxels in four error-feedback chains of 8 (x = 8k + j, k = 0..3): chains
// 0 / 1 and 2 / 3 advance together as two packed pairs, so each step has two
// independent dependency chains and a run takes 8 steps instead of 16.  Used
// for the intermediate field of the fused y + x kernel, which the x MMAs
// consume at once (its rounding noise, high-pass within 8 voxels, is removed
// by the x convolution that follows).  d[j] holds voxels j (low) and 8 + j
// (high); d[8 + j] holds 16 + j and 24 + j.  No masking: a run outside the
// volume holds zeros, which round to zeros.
template <typename S>
__device__ __forceinline__ void narrow32_quads(const float (&a)[32], float scale, bool ef, uint32_t (&d)[16]) {
    float2 c0 = make_float2(0.0f, 0.0f), c1 = make_float2(0.0f, 0.0f);
    const float2 s2 = make_float2(scale, scale), m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
    for (int j = 0; j < 8; j++) {
        float2 w0 = make_float2(a[j], a[8 + j]), w1 = make_float2(a[16 + j], a[24 + j]);
        w0 = ef ? __ffma2_rn(w0, s2, c0) : __fmul2_rn(w0, s2);
        w1 = ef ? __ffma2_rn(w1, s2, c1) : __fmul2_rn(w1, s2);
        const uint32_t q0 = Pair16<S>::cvt(w0.x, w0.y), q1 = Pair16<S>::cvt(w1.x, w1.y);
        if (ef) {
            c0 = __ffma2_rn(Pair16<S>::widen(q0), m1, w0);
            c1 = __ffma2_rn(Pair16<S>::widen(q1), m1, w1);
        }
        d[j] = q0;
        d[8 + j] = q1;
    }
}

// Two 32-voxel runs as narrow32_quads<S> each (a[0..31] -> d0,
// a[32..63] -> d1), their chains interleaved: four independent chains per step.
template <typename S>
__device__ __forceinline__ void narrow64_quads(const float (&a)[64], float scale, bool ef, uint32_t (&d0)[16],
                                               uint32_t (&d1)[16]) {
    float2 c[4] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
    const float2 s2 = make_float2(scale, scale), m1 = make_float2(-1.0f, -1.0f);
#pragma unroll
    for (int j = 0; j < 8; j++) {
#pragma unroll
        for (int h = 0; h < 4; h++) {  // h: run h / 2, chains pair h % 2
            const int b = 32 * (h >> 1) + 16 * (h & 1);
            float2 w = make_float2(a[b + j], a[b + 8 + j]);
            w = ef ? __ffma2_rn(w, s2, c[h]) : __fmul2_rn(w, s2);
            const uint32_t q = Pair16<S>::cvt(w.x, w.y);
            if (ef) c[h] = __ffma2_rn(Pair16<S>::widen(q), m1, w);
            ((h >> 1) ? d1 : d0)[8 * (h & 1) + j] = q;
        }
    }
}

// narrow32_quads' words -> pairs of neighbours: o[i] = voxels (2i, 2i + 1).
__device__ __forceinline__ void quads_to_adjacent(const uint32_t (&d)[16], uint32_t (&o)[16]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        o[i] = __byte_perm(d[2 * i], d[2 * i + 1], 0x5410);           // voxels 2i, 2i + 1 (chain 0)
        o[4 + i] = __byte_perm(d[2 * i], d[2 * i + 1], 0x7632);       // 8 + 2i, 9 + 2i (chain 1)
        o[8 + i] = __byte_perm(d[8 + 2 * i], d[9 + 2 * i], 0x5410);   // 16 + 2i, 17 + 2i (chain 2)
        o[12 + i] = __byte_perm(d[8 + 2 * i], d[9 + 2 * i], 0x7632);  // 24 + 2i, 25 + 2i (chain 3)
    }
}

// Pairs (j, 16 + j) -> pairs of neighbours: o[i] = voxels (2i, 2i + 1), i < 16.
__device__ __forceinline__ void pairs_to_adjacent(const uint32_t (&d)[16], uint32_t (&o)[16]) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
        o[i] = __byte_perm(d[2 * i], d[2 * i + 1], 0x5410);
        o[8 + i] = __byte_perm(d[2 * i], d[2 * i + 1], 0x7632);
    }
}

// Packs 8 consecutive 16-bit values into a 16-byte vector.
__device__ __forceinline__ uint4 pack8(const uint16_t *q) {
    uint4 u;
    u.x = q[0] | ((uint32_t) q[1] << 16);
    u.y = q[2] | ((uint32_t) q[3] << 16);
    u.z = q[4] | ((uint32_t) q[5] << 16);
    u.w = q[6] | ((uint32_t) q[7] << 16);
    return u;
}

// Stores 32 consecutive 16-bit values (count of them valid) at dst.
__device__ __forceinline__ void store32_u16(uint16_t *dst, const uint16_t (&q)[32], int count) {
    if (count == 32) {
#pragma unroll
        for (int i = 0; i < 32; i += 8) *reinterpret_cast<uint4 *>(dst + i) = pack8(q + i);
    } else {
#pragma unroll
        for (int i = 0; i < 32; i++)
            if (i < count) dst[i] = q[i];
    }
}

// Last-repetition x-pass epilogue of one thread: 32 consecutive voxels of
// one row from x = xb -- re-illumination, then the uint16 output and the FP32
// field (either may be NULL).  Requires nx % 8 == 0 and 16-byte aligned outputs.
__device__ __forceinline__ void contig_final32(const float (&h)[32], uint32_t m, int64_t row, int64_t rows,
                                               int64_t nx, int64_t xb, float scale, uint16_t *out_u16,
                                               float *field_out) {
    if (row >= rows || xb >= nx) return;
    const int count = nx - xb < 32 ? (int) (nx - xb) : 32;
    const int64_t idx = row * nx + xb;
    float v[32];
    uint16_t q[32];
#pragma unroll
    for (int i = 0; i < 32; i++) {
        v[i] = ((m >> i) & 1u) ? 1.0f : h[i] * scale;
        q[i] = quantise_u16(v[i]);
    }
    if (out_u16) store32_u16(out_u16 + idx, q, count);
    if (field_out) {
        if (count == 32) {
#pragma unroll
            for (int i = 0; i < 32; i += 4)
                *reinterpret_cast<float4 *>(field_out + idx + i) = make_float4(v[i], v[i + 1], v[i + 2], v[i + 3]);
        } else {
#pragma unroll
            for (int i = 0; i < 32; i++)
                if (i < count) field_out[idx + i] = v[i];
        }
    }
}

// Mask flags of up to 32 voxels of a row (bit q = voxel idx + q), with a
// 2 x 16-byte vector read for aligned full uint8 chunks.
template <int FMT>
__device__ __forceinline__ uint32_t row_mask32(const void *m, int64_t idx, int count, int64_t n) {
    if (FMT == MAXI_MASK_U8 && count == 32 && ((reinterpret_cast<uintptr_t>(m) + idx) & 15) == 0) {
        const uint4 *p = reinterpret_cast<const uint4 *>(static_cast<const uint8_t *>(m) + idx);
        const uint4 a = __ldg(p), b = __ldg(p + 1);
        const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        uint32_t r = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
#pragma unroll
            for (int by = 0; by < 4; by++) r |= (uint32_t) (((w[q] >> (8 * by)) & 0xffu) != 0u) << (q * 4 + by);
        }
        return r;
    }
    return mask32<FMT>(m, idx, count, n);
}

}  // namespace tc
}  // namespace maxi
