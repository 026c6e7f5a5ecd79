// Host-side helpers shared by the C ABI translation units: error state,
// argument validation, integer arithmetic.
#pragma once

#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <algorithm>
#include <string>

#include "../../include/maxibone_diffusion.h"

namespace maxi {

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
inline int64_t round_up(int64_t a, int64_t b) { return ceil_div(a, b) * b; }

// Per-thread message for maxi_last_error().
inline std::string &last_error_ref() {
    static thread_local std::string msg;
    return msg;
}
inline const char *last_error_cstr() { return last_error_ref().c_str(); }
inline void clear_error() { last_error_ref().clear(); }

inline int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    last_error_ref() = buf;
    return code;
}

// Per-thread record of the kernel families (MAXI_PATH_* bits) the last
// diffusion call of this thread enqueued, for maxi_last_path().
inline int &last_path_ref() {
    static thread_local int path = 0;
    return path;
}
inline void note_path(int bits) { last_path_ref() |= bits; }

inline int set_cuda_error(cudaError_t e, const char *what) {
    const int code = (e == cudaErrorMemoryAllocation) ? MAXI_ERR_OUT_OF_MEMORY : MAXI_ERR_CUDA;
    return set_error(code, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
}

inline int require_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return set_error(MAXI_ERR_NO_DEVICE, "no CUDA device is visible");
    }
    return MAXI_OK;
}

// Checks shared by every diffusion entry point.  The reference does none of
// these (shape mismatch and even kernels are undefined behaviour there,
// src/pybind/diffusion-pybind.cc:27-53); here they are errors.
inline int validate_common(const void *mask, int64_t nz, int64_t ny, int64_t nx, const float *kernel,
                           int64_t kernel_size, int64_t reps, int64_t max_radius = 1024) {
    if (!mask) return set_error(MAXI_ERR_INVALID_ARGUMENT, "mask is NULL");
    if (!kernel) return set_error(MAXI_ERR_INVALID_ARGUMENT, "kernel is NULL");
    if (nz <= 0 || ny <= 0 || nx <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "shape (%lld, %lld, %lld) has an empty axis",
                         (long long) nz, (long long) ny, (long long) nx);
    if (nz > (int64_t(1) << 40) / ny / nx)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "volume of more than 2^40 voxels");
    if (kernel_size <= 0 || kernel_size % 2 == 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "kernel length %lld is not odd and positive",
                         (long long) kernel_size);
    if (kernel_size / 2 > max_radius)
        return set_error(MAXI_ERR_UNSUPPORTED, "kernel radius %lld exceeds the supported %lld",
                         (long long) (kernel_size / 2), (long long) max_radius);
    if (reps < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "negative repetition count %lld", (long long) reps);
    return MAXI_OK;
}

// Frees the sphere-morphology scratch kept between calls (morphology.cu).
void release_morphology_scratch();

}  // namespace maxi
