// Unrolled CUDA-core repetition loop, instantiated per field storage type in
// passes_<type>.cu so that the instantiations compile in parallel.
#pragma once

#include "common.cuh"
#include "host_util.h"

namespace maxi {

struct Volume {
    int64_t nz, ny, nx;
    int64_t n() const { return nz * ny * nx; }
};

// Packs a uint8 mask into uint32 words, MSB first (bitpack.cu).  keep_bit0:
// the reference encode's `mask & 1`; otherwise the diffusion's `mask > 0`.
cudaError_t launch_bitpack_encode(const uint8_t *mask, int64_t n, uint32_t *packed, bool keep_bit0, cudaStream_t st);

// field <- mask > 0 ? 1 : 0 in the storage type (rep-0 input).
template <typename S>
cudaError_t launch_init_field(const void *mask, int mask_fmt, S *field, int64_t n, cudaStream_t st);

// Smallest radius with an unrolled instantiation that is >= r, or -1.
int radius_bucket(int r);

// Options of one repetition loop beyond the volume and its buffers.
struct RunOpts {
    // Out-of-core slabs: repetition k works on planes [k*shrink_lo, nz -
    // k*shrink_hi) only -- the planes that can still reach the slab's core; the
    // bit-packed mask must then have (ny*nx) % 32 == 0.
    int64_t shrink_lo = 0, shrink_hi = 0;
    // Start from this FP32 field (device or mapped host memory, nz*ny*nx
    // values) instead of the mask (out-of-core exchange rounds).
    const float *init_field = nullptr;
    // The last repetition waits for this event before it starts (lets the
    // caller overlap a copy out of the output buffers with the earlier ones).
    cudaEvent_t final_wait = nullptr;
};

// Runs `reps` repetitions (reps >= 1) of the unrolled passes: buf0 receives
// the initial field, buf0/buf1 ping-pong, the last x pass writes out_u16 and
// field_out (either may be NULL).
// flags: MAXI_FLAG_* bits (NO_TENSOR_CORES and NEAREST_ROUNDING apply to the
// 16-bit storage types).
template <typename S>
cudaError_t dispatch_unrolled(const Volume &v, const void *mask, int mask_fmt, const float *kernel, int radius,
                              int64_t reps, S *b0, S *b1, uint16_t *out_u16, float *field_out, int32_t flags,
                              cudaStream_t st, const RunOpts &o = RunOpts{});

// maxi_diffusion_device() with the RunOpts of an out-of-core slab.
int diffusion_device_shrinking(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                               const float *kernel, int64_t kernel_size, int64_t repititions, uint16_t *output,
                               void *field_out, int32_t field_type, int32_t flags, void *workspace,
                               int64_t workspace_bytes, void *stream, const RunOpts &o);

}  // namespace maxi
