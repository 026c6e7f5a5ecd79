// Host orchestration and C ABI of the mask-diffusion library.
//
// The reference entry points this file replaces:
//   NS::diffusion_in_memory  src/lib/cpp/include/diffusion.hh:36
//                            (CPU body src/lib/cpp/cpu/diffusion.cc:339-374,
//                             OpenACC body src/lib/cpp/gpu/diffusion.cc:758-806)
//   python_api::diffusion_in_memory  src/pybind/diffusion-pybind.cc:27-53
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <map>
#include <mutex>
#include <atomic>

#include "common.cuh"
#include "passes.cuh"
#include "host_util.h"
#include "host_copy.h"
#include "unrolled.h"
#include "profiler.h"
#include "tc_pass.h"
#include "tc_batch.h"

namespace maxi {

// Generic passes: FP64 form, reference rounding, radii beyond the unrolled set.
template <typename S, bool EXACT, int MF>
static cudaError_t run_generic_fmt(const Volume &v, const void *mask, const float *kernel, int radius,
                                   int64_t reps, S *b0, S *b1, uint16_t *out_u16, void *field_out,
                                   const RunOpts &o, cudaStream_t st) {
    using Acc = typename FieldIO<S>::Acc;
    auto *taps = new GenericTaps<Acc>();
    for (int i = 0; i < 2 * radius + 1; i++) taps->k[i] = (Acc) kernel[i];
    const int64_t n = v.n();
    const int threads = 256;
    const int64_t blocks = ceil_div(n, threads);
    {
        ProfScope ps(MAXI_KERNEL_INIT, st);
        if (o.init_field)
            field_from_f32<S><<<std::min<int64_t>(blocks, 148 * 64), threads, 0, st>>>(o.init_field, b0, n);
        else
            mask_to_field<S, MF, false><<<std::min<int64_t>(blocks, 148 * 64), threads, 0, st>>>(mask, b0, nullptr, nullptr, n);
    }
    for (int64_t rep = 0; rep < reps; rep++) {
        if (o.final_wait && rep + 1 == reps) {
            const cudaError_t e = cudaStreamWaitEvent(st, o.final_wait, 0);
            if (e != cudaSuccess) {
                delete taps;
                return e;
            }
        }
        {
            ProfScope ps(MAXI_KERNEL_Z, st);
            generic_pass<S, EXACT, false, MF, false><<<blocks, threads, 0, st>>>(b0, b1, mask, nullptr, nullptr, n, v.nz, v.ny * v.nx, radius, *taps);
        }
        {
            ProfScope ps(MAXI_KERNEL_Y, st);
            generic_pass<S, EXACT, false, MF, false><<<blocks, threads, 0, st>>>(b1, b0, mask, nullptr, nullptr, n, v.ny, v.nx, radius, *taps);
        }
        if (rep + 1 < reps) {
            ProfScope ps(MAXI_KERNEL_X, st);
            generic_pass<S, EXACT, true, MF, false><<<blocks, threads, 0, st>>>(b0, b1, mask, nullptr, nullptr, n, v.nx, 1, radius, *taps);
            std::swap(b0, b1);
        } else {
            ProfScope ps(MAXI_KERNEL_X_FINAL, st);
            generic_pass<S, EXACT, true, MF, true><<<blocks, threads, 0, st>>>(b0, b1, mask, out_u16, field_out, n, v.nx, 1, radius, *taps);
        }
    }
    delete taps;
    return cudaGetLastError();
}

template <typename S, bool EXACT>
static cudaError_t run_generic(const Volume &v, const void *mask, int mask_fmt, const float *kernel, int radius,
                               int64_t reps, S *b0, S *b1, uint16_t *out_u16, void *field_out, const RunOpts &o,
                               cudaStream_t st) {
    if (mask_fmt == MAXI_MASK_U8)
        return run_generic_fmt<S, EXACT, MAXI_MASK_U8>(v, mask, kernel, radius, reps, b0, b1, out_u16, field_out, o, st);
    return run_generic_fmt<S, EXACT, MAXI_MASK_BITPACKED>(v, mask, kernel, radius, reps, b0, b1, out_u16, field_out, o, st);
}

template <typename S>
static cudaError_t zero_reps(const Volume &v, const void *mask, int mask_fmt, uint16_t *out_u16, void *field_out,
                             cudaStream_t st) {
    const int64_t n = v.n();
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), 148 * 64);
    ProfScope ps(MAXI_KERNEL_X_FINAL, st);
    if (mask_fmt == MAXI_MASK_U8)
        mask_to_field<S, MAXI_MASK_U8, true><<<blocks, 256, 0, st>>>(mask, nullptr, out_u16, field_out, n);
    else
        mask_to_field<S, MAXI_MASK_BITPACKED, true><<<blocks, 256, 0, st>>>(mask, nullptr, out_u16, field_out, n);
    return cudaGetLastError();
}

static size_t field_bytes(int32_t ft) {
    switch (ft) {
    case MAXI_FIELD_F32: return 4;
    case MAXI_FIELD_BF16: return 2;
    case MAXI_FIELD_F16: return 2;
    case MAXI_FIELD_F64: return 8;
    default: return 0;
    }
}

// Two field buffers plus the bit-packed copy of a uint8 mask (the passes read
// the mask as 1 bit per voxel).
static int64_t workspace_bytes_for(int64_t n, int32_t ft) {
    return 2 * round_up((int64_t) field_bytes(ft) * n, 256) + round_up(ceil_div(n, 32) * 4, 256);
}

template <typename S>
static cudaError_t run_typed(const Volume &v, const void *mask, int mask_fmt, const float *kernel, int radius,
                             int64_t reps, uint16_t *out_u16, void *field_out, int32_t flags, char *ws,
                             cudaStream_t st, const RunOpts &o) {
    if (reps == 0) return zero_reps<S>(v, mask, mask_fmt, out_u16, field_out, st);
    S *b0 = reinterpret_cast<S *>(ws);
    S *b1 = reinterpret_cast<S *>(ws + round_up((int64_t) sizeof(S) * v.n(), 256));
    constexpr bool is_f64 = std::is_same<S, double>::value;
    const bool exact = (flags & MAXI_FLAG_REFERENCE_ROUNDING) != 0;
    if (is_f64 || exact || radius_bucket(radius) < 0) {
        note_path(MAXI_PATH_GENERIC);
        if (exact) return run_generic<S, true>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16, field_out, o, st);
        return run_generic<S, false>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16, field_out, o, st);
    }
    if constexpr (!is_f64) {
        uint32_t *packed = reinterpret_cast<uint32_t *>(ws + 2 * round_up((int64_t) sizeof(S) * v.n(), 256));
        if (mask_fmt == MAXI_MASK_U8) {
            // Read the mask as 1 bit per voxel in every x pass: pack it once.
            cudaError_t e = launch_bitpack_encode(static_cast<const uint8_t *>(mask), v.n(), packed, false, st);
            if (e != cudaSuccess) return e;
            mask = packed;
            mask_fmt = MAXI_MASK_BITPACKED;
        } else if (flags & MAXI_FLAG_MASK_FROM_FIELD) {
            // The mask is rewritten every repetition: work on a copy, never the caller's.
            cudaError_t e = cudaMemcpyAsync(packed, mask, ceil_div(v.n(), 32) * 4, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return e;
            mask = packed;
        }
        return dispatch_unrolled<S>(v, mask, mask_fmt, kernel, radius, reps, b0, b1, out_u16,
                                    static_cast<float *>(field_out), flags, st, o);
    }
    return cudaErrorInvalidValue;
}

// Device buffers of the host entry point (one per device, grow-only): freed
// before the call returns unless the caller asked to keep them between calls
// (maxi_keep_device_buffers), so that repeated calls do not map and unmap
// gigabytes each time.
struct DeviceCache {
    std::mutex mu;
    void *buf = nullptr;
    int64_t bytes = 0;
    cudaStream_t stream = nullptr;
};
static std::mutex g_cache_mu;
static std::map<int, DeviceCache *> g_caches;
// Whether maxi_diffusion_in_memory() keeps its device buffers after it
// returns (maxi_keep_device_buffers); off by default, as the reference frees
// its working buffers before returning (src/lib/cpp/cpu/diffusion.cc:371-373).
static std::atomic<int> g_keep_buffers{0};

static void cache_drop(DeviceCache *c) {
    if (!c->buf) return;
    cudaStreamSynchronize(c->stream);
    cudaFree(c->buf);
    c->buf = nullptr;
    c->bytes = 0;
}

static int device_cache(DeviceCache **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    std::lock_guard<std::mutex> lk(g_cache_mu);
    DeviceCache *&c = g_caches[dev];
    if (!c) {
        c = new DeviceCache();
        if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
            return set_cuda_error(e, "stream creation");
    }
    *out = c;
    return MAXI_OK;
}

static int cache_reserve(DeviceCache *c, int64_t bytes) {
    if (c->bytes >= bytes) return MAXI_OK;
    cache_drop(c);
    if (cudaMalloc(&c->buf, bytes) != cudaSuccess) {
        cudaGetLastError();
        c->buf = nullptr;
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %lld bytes on the device", (long long) bytes);
    }
    c->bytes = bytes;
    return MAXI_OK;
}

static void release_device_caches() {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (auto &kv : g_caches) {
        std::lock_guard<std::mutex> lk2(kv.second->mu);
        cache_drop(kv.second);
    }
}

}  // namespace maxi

using namespace maxi;

extern "C" int maxi_diffusion_out_of_core_ex(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                                             int64_t slab_z, const float *kernel, int64_t kernel_size,
                                             int64_t repititions, uint16_t *output, int32_t field_type,
                                             int32_t flags, int verbose);

extern "C" {

const char *maxi_version(void) { return "maxibone_b200 diffusion 0.1 (sm_100a)"; }

const char *maxi_last_error(void) { return last_error_cstr(); }

int maxi_last_path(void) { return last_path_ref(); }

int maxi_tensor_core_status(void) {
    clear_error();
    const int a = tc::tc_read_and_clear_error(), b = tc::tc_batch_read_and_clear_error();
    const int v = (a < 0 || b < 0) ? -1 : (a ? a : b);
    if (v < 0) return set_error(MAXI_ERR_CUDA, "could not read the tensor-core error word");
    if (v > 0) return set_error(MAXI_ERR_CUDA, "a tensor-core pass timed out waiting (code %d)", v);
    return MAXI_OK;
}

int maxi_tensor_core_taps(const float *kernel, int64_t kernel_size, int32_t field_type, uint16_t *taps,
                          float *inv_scale) {
    clear_error();
    if (!kernel || !taps || !inv_scale) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (kernel_size < 1 || kernel_size % 2 == 0 || kernel_size > 2 * tc::kTcMaxRadiusWide + 1)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "kernel_size must be odd and at most %d",
                         2 * tc::kTcMaxRadiusWide + 1);
    if (field_type != MAXI_FIELD_BF16 && field_type != MAXI_FIELD_F16)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "field_type must be MAXI_FIELD_BF16 or MAXI_FIELD_F16");
    const bool bf16 = field_type == MAXI_FIELD_BF16;
    // the base scale of the passes' taps (fill_pass_taps): FP16 taps are lifted into the normal range
    const float s = tc::tc_round_taps_scaled(kernel, (int) (kernel_size / 2), bf16, bf16 ? 1.0f : 1024.0f, taps);
    *inv_scale = 1.0f / s;
    return MAXI_OK;
}

int64_t maxi_diffusion_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t field_type) {
    if (nz <= 0 || ny <= 0 || nx <= 0 || field_bytes(field_type) == 0) return -1;
    return workspace_bytes_for(nz * ny * nx, field_type);
}

int maxi_diffusion_device(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                          const float *kernel, int64_t kernel_size, int64_t repititions,
                          uint16_t *output, void *field_out, int32_t field_type, int32_t flags,
                          void *workspace, int64_t workspace_bytes, void *stream) {
    return diffusion_device_shrinking(mask, mask_format, nz, ny, nx, kernel, kernel_size, repititions, output,
                                      field_out, field_type, flags, workspace, workspace_bytes, stream, RunOpts{});
}

int maxi_diffusion_device_ex(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                             const float *kernel, int64_t kernel_size, int64_t repititions, uint16_t *output,
                             void *field_out, int32_t field_type, int32_t flags, void *workspace,
                             int64_t workspace_bytes, void *stream, const float *init_field, int64_t shrink_lo,
                             int64_t shrink_hi) {
    if (shrink_lo < 0 || shrink_hi < 0) {
        clear_error();
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "negative window shrink");
    }
    if (init_field && (reinterpret_cast<uintptr_t>(init_field) & 3) != 0) {
        clear_error();
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "init_field is not 4-byte aligned");
    }
    if (init_field && repititions == 0) {
        clear_error();
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "a run continued from a field needs at least one repetition");
    }
    RunOpts o;
    o.shrink_lo = shrink_lo;
    o.shrink_hi = shrink_hi;
    o.init_field = init_field;
    return diffusion_device_shrinking(mask, mask_format, nz, ny, nx, kernel, kernel_size, repititions, output,
                                      field_out, field_type, flags, workspace, workspace_bytes, stream, o);
}

}  // extern "C"

int maxi::diffusion_device_shrinking(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                                     const float *kernel, int64_t kernel_size, int64_t repititions,
                                     uint16_t *output, void *field_out, int32_t field_type, int32_t flags,
                                     void *workspace, int64_t workspace_bytes, void *stream, const RunOpts &opts) {
    clear_error();
    int rc = validate_common(mask, nz, ny, nx, kernel, kernel_size, repititions);
    if (rc) return rc;
    if (mask_format != MAXI_MASK_U8 && mask_format != MAXI_MASK_BITPACKED)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "unknown mask_format %d", mask_format);
    if (field_bytes(field_type) == 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "unknown field_type %d", field_type);
    if ((flags & MAXI_FLAG_REFERENCE_ROUNDING) && field_type != MAXI_FIELD_F32)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "reference rounding is defined for the FP32 field only");
    if ((flags & MAXI_FLAG_MASK_FROM_FIELD) &&
        (field_type != MAXI_FIELD_F32 || (flags & MAXI_FLAG_REFERENCE_ROUNDING) || kernel_size / 2 > 128))
        return set_error(MAXI_ERR_UNSUPPORTED,
                         "the rebuilt-mask semantics are served for the FP32 field with the fast passes (radius <= 128)");
    if (!output && !field_out)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "neither output nor field_out given");
    // The passes read the workspace's field buffers with 16-byte vector and
    // TMA loads, and a bit-packed mask as 32-bit words: misaligned pointers
    // would fault on the device, so they are rejected here.
    if (workspace && (reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "workspace is not 256-byte aligned");
    if (mask_format == MAXI_MASK_BITPACKED && (reinterpret_cast<uintptr_t>(mask) & 3) != 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "a bit-packed mask must be 4-byte aligned");
    if ((rc = require_device())) return rc;
    last_path_ref() = 0;

    const Volume v{nz, ny, nx};
    const int radius = (int) (kernel_size / 2);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char *ws = static_cast<char *>(workspace);
    // A 16-bit field on a shape the tensor-core passes do not take (nx not a
    // multiple of 8, nx < 64) would run the 16-bit CUDA-core passes, which are
    // slower than the FP32 form as well as less accurate: such a request runs
    // the FP32 form instead when the workspace allows it (reported by
    // maxi_last_path()).  MAXI_FLAG_NO_TENSOR_CORES keeps the 16-bit passes.
    int32_t run_type = field_type;
    if ((field_type == MAXI_FIELD_BF16 || field_type == MAXI_FIELD_F16) && !(flags & MAXI_FLAG_NO_TENSOR_CORES) &&
        repititions > 0 && radius_bucket(radius) >= 0 && !tc::tc_supported(radius, nz, ny, nx) &&
        (!ws || workspace_bytes >= workspace_bytes_for(v.n(), MAXI_FIELD_F32))) {
        run_type = MAXI_FIELD_F32;
        note_path(MAXI_PATH_FP32_FALLBACK);
    }
    const int64_t need = workspace_bytes_for(v.n(), run_type);
    bool owned = false;
    if (repititions > 0) {
        if (ws && workspace_bytes < need)
            return set_error(MAXI_ERR_INVALID_ARGUMENT, "workspace of %lld bytes is smaller than the %lld needed",
                             (long long) workspace_bytes, (long long) need);
        if (!ws) {
            if (cudaMallocAsync(reinterpret_cast<void **>(&ws), need, st) != cudaSuccess) {
                cudaGetLastError();
                return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %lld bytes of device workspace",
                                 (long long) need);
            }
            owned = true;
        }
    }
    // Plane windows start at multiples of ny*nx voxels: keep them on whole
    // 32-bit words of the bit-packed mask (and 16-byte aligned for TMA).
    RunOpts o = opts;
    if ((ny * nx) % 32 != 0 || o.shrink_lo < 0 || o.shrink_hi < 0 || run_type == MAXI_FIELD_F64)
        o.shrink_lo = o.shrink_hi = 0;
    cudaError_t e;
    switch (run_type) {
    case MAXI_FIELD_F32: e = run_typed<float>(v, mask, mask_format, kernel, radius, repititions, output, field_out, flags, ws, st, o); break;
    case MAXI_FIELD_BF16: e = run_typed<__nv_bfloat16>(v, mask, mask_format, kernel, radius, repititions, output, field_out, flags, ws, st, o); break;
    case MAXI_FIELD_F16: e = run_typed<__half>(v, mask, mask_format, kernel, radius, repititions, output, field_out, flags, ws, st, o); break;
    default: e = run_typed<double>(v, mask, mask_format, kernel, radius, repititions, output, field_out, flags, ws, st, o); break;
    }
    if (owned) cudaFreeAsync(ws, st);
    if (e != cudaSuccess) return set_cuda_error(e, "diffusion launch");
    return MAXI_OK;
}

extern "C" {

int maxi_diffusion_in_memory(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                             const float *kernel, int64_t kernel_size, int64_t repititions,
                             uint16_t *output, int verbose) {
    clear_error();
    int rc = validate_common(voxels, nz, ny, nx, kernel, kernel_size, repititions);
    if (rc) return rc;
    if (!output) return set_error(MAXI_ERR_INVALID_ARGUMENT, "output is NULL");
    if ((rc = require_device())) return rc;
    const int64_t n = nz * ny * nx;
    const int64_t need = workspace_bytes_for(n, MAXI_FIELD_F32);
    const int64_t mask_off = 0, out_off = round_up(n, 256), ws_off = out_off + round_up(2 * n, 256);
    const int64_t total = ws_off + need;
    if (verbose >= 1)
        printf("Diffusion: shape (%lld, %lld, %lld), kernel size %lld, %lld repetitions, FP32 field on the GPU\n",
               (long long) nz, (long long) ny, (long long) nx, (long long) kernel_size, (long long) repititions);
    DeviceCache *cache = nullptr;
    if ((rc = device_cache(&cache))) return rc;
    std::lock_guard<std::mutex> lk(cache->mu);
    if ((rc = cache_reserve(cache, total))) {
        // Larger than the device: the reference's pybind module sends such volumes to
        // its out-of-core form (src/pybind/diffusion-pybind.cc:40-45); do the same,
        // with the slab depth (and exchange rounds, for large R x radius) chosen
        // from the free device memory.
        if (verbose >= 1) printf("Volume exceeds device memory: out-of-core form\n");
        clear_error();
        return maxi_diffusion_out_of_core_ex(voxels, nz, ny, nx, 0, kernel, kernel_size, repititions, output,
                                             MAXI_FIELD_F32, 0, verbose);
    }
    char *base = static_cast<char *>(cache->buf);
    uint8_t *d_mask = reinterpret_cast<uint8_t *>(base + mask_off);
    uint16_t *d_out = reinterpret_cast<uint16_t *>(base + out_off);
    cudaStream_t st = cache->stream;
    // Pageable caller buffers of some size go through pinned staging with
    // several host threads; pinned ones are copied directly.
    const int64_t stage_min = int64_t(64) << 20;
    const bool stage_in = n >= stage_min && host_pageable(voxels);
    const bool stage_out = 2 * n >= stage_min && host_pageable(output);
    cudaError_t e = stage_in ? copy_to_device_staged(d_mask, voxels, n, st)
                             : cudaMemcpyAsync(d_mask, voxels, n, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        rc = maxi_diffusion_device(d_mask, MAXI_MASK_U8, nz, ny, nx, kernel, kernel_size, repititions, d_out, nullptr,
                                   MAXI_FIELD_F32, 0, base + ws_off, need, st);
        if (rc) {
            if (!g_keep_buffers.load()) cache_drop(cache);
            return rc;
        }
        e = stage_out ? copy_to_host_staged(output, d_out, 2 * n, st)
                      : cudaMemcpyAsync(output, d_out, 2 * n, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (!g_keep_buffers.load()) cache_drop(cache);
    if (e != cudaSuccess) return set_cuda_error(e, "in-memory diffusion");
    if (verbose >= 1) printf("Diffusion is complete!\n");
    return MAXI_OK;
}

int maxi_keep_device_buffers(int keep) {
    clear_error();
    g_keep_buffers.store(keep ? 1 : 0);
    if (!keep) release_device_caches();
    return MAXI_OK;
}

int maxi_release_cached_memory(void) {
    clear_error();
    release_device_caches();
    release_morphology_scratch();
    return MAXI_OK;
}

}  // extern "C"
