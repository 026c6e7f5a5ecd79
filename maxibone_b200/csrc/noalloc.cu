// Allocation-free entry point: the FP32 diffusion with its two field buffers
// taken from a fixed array compiled into this library instead of from
// cudaMalloc.
//
// Who needs it: callers that must not allocate device memory while they run --
// for example a host that has handed the whole device heap to its own
// sub-allocator and forbids other allocations, a process that has to stay
// within a fixed memory budget decided at start-up, or real-time code where an
// allocation (which can synchronise the device or fail under memory pressure)
// is not acceptable in the middle of its work.  They pass the mask, the output
// and optionally the field output; the library itself allocates nothing.
//
// Limits and rules of use:
//   * at most kNoAllocMaxVoxels voxels per call (e.g. 256 x 256 x 128); larger
//     volumes are rejected with MAXI_ERR_INVALID_ARGUMENT before any GPU work;
//   * the array (2 * kNoAllocMaxVoxels floats = 64 MiB) stays reserved until the
//     process exits on every GPU where this library's device code is loaded.
//     With CUDA's default lazy module loading that is the GPUs that use this
//     entry point; with eager loading (CUDA_MODULE_LOADING=EAGER) it is every
//     GPU on which the process creates a context while the library is loaded;
//   * the first call on each device looks up the array's device address with
//     cudaGetSymbolAddress (which may load this part of the library), so make
//     that first call before any stream capture starts;
//   * all calls share the one array, and the array keeps whatever the last call
//     left in it; nothing needs to start at zero because every repetition
//     overwrites both buffers completely before reading them.  Two calls whose
//     GPU work overlaps -- on different streams or from different host threads
//     without ordering between them -- race on the array and give wrong results:
//     serialise them (one stream, or events).
#include <mutex>

#include "common.cuh"
#include "host_util.h"
#include "unrolled.h"

namespace maxi {

constexpr int64_t kNoAllocMaxVoxels = int64_t(1) << 23;  // 8,388,608 voxels
constexpr int kNoAllocMaxDevices = 64;

// Two FP32 field buffers of kNoAllocMaxVoxels each.
static __device__ __align__(256) float g_noalloc_scratch[2 * kNoAllocMaxVoxels];

namespace {
std::mutex g_noalloc_mu;
float *g_noalloc_ptr[kNoAllocMaxDevices] = {};
}  // namespace

// Device address of the scratch array for the current device.  On the host
// the symbol `g_noalloc_scratch` names a host-side stand-in, not device
// memory, so it must never be passed to a kernel directly.
static int noalloc_scratch(float **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDevice");
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(MAXI_ERR_UNSUPPORTED, "device ordinal %d above %d", dev, kNoAllocMaxDevices - 1);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return set_cuda_error(e, "cudaGetSymbolAddress of the no-alloc scratch array");
        g_noalloc_ptr[dev] = static_cast<float *>(p);
    }
    *out = g_noalloc_ptr[dev];
    return MAXI_OK;
}

}  // namespace maxi

using namespace maxi;

extern "C" int maxi_diffusion_device_noalloc(const void *mask, int32_t mask_format, int64_t nz, int64_t ny,
                                             int64_t nx, const float *kernel, int64_t kernel_size,
                                             int64_t repititions, uint16_t *output, float *field_out,
                                             void *stream) {
    clear_error();
    int rc = validate_common(mask, nz, ny, nx, kernel, kernel_size, repititions, 128);
    if (rc) return rc;
    if (mask_format != MAXI_MASK_U8 && mask_format != MAXI_MASK_BITPACKED)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "unknown mask_format %d", mask_format);
    if (!output && !field_out) return set_error(MAXI_ERR_INVALID_ARGUMENT, "neither output nor field_out given");
    if (mask_format == MAXI_MASK_BITPACKED && (reinterpret_cast<uintptr_t>(mask) & 3) != 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "a bit-packed mask must be 4-byte aligned");
    const int64_t n = nz * ny * nx;
    if (n > kNoAllocMaxVoxels)
        return set_error(MAXI_ERR_INVALID_ARGUMENT,
                         "volume of %lld voxels exceeds the no-alloc limit of %lld voxels",
                         (long long) n, (long long) kNoAllocMaxVoxels);
    if (repititions == 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "the no-alloc entry point needs at least one repetition");
    if ((rc = require_device())) return rc;
    float *scratch = nullptr;
    if ((rc = noalloc_scratch(&scratch))) return rc;
    last_path_ref() = 0;
    const Volume v{nz, ny, nx};
    cudaError_t e = dispatch_unrolled<float>(v, mask, mask_format, kernel, (int) (kernel_size / 2), repititions,
                                             scratch, scratch + kNoAllocMaxVoxels, output, field_out, 0,
                                             static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return set_cuda_error(e, "no-alloc diffusion launch");
    return MAXI_OK;
}
