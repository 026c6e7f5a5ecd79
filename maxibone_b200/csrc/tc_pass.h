// Host interface of the tensor-core (tcgen05) passes for 16-bit field storage.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace maxi {
namespace tc {

// Largest kernel radius of the batched tensor-core passes and of the x pass in
// its direct form (its shared-memory Toeplitz, K = 128 + 2 * 32 rows of both
// halves, and a 2-stage tile ring must fit shared memory).
constexpr int kTcMaxRadius = 32;
// Largest radius of the single-volume tensor-core passes: the z / y passes
// hold the Toeplitz halves in tensor memory (192 columns each at radius 128,
// next to 64-column accumulators) and load K = 128 + 2r rows as two TMA
// boxes; the x pass above radius 32 runs in its transposed form.
constexpr int kTcMaxRadiusWide = 128;

// Smallest radius served by one 16-bit coefficient set (tc_round_taps_scaled):
// the set's scale is searched so that its sum matches the kernel's (to 2e-7 at
// sigma 1, 2e-8 from sigma 2), which keeps small-sigma kernels within the
// error bound too (BF16, sigma 2, R = 50: 1.3e-3 over the batch's volumes; a
// set at scale 1 gave 2.4e-3).
// Below radius 4 the 16-bit stores round to nearest and the passes use the
// high + low halves.
constexpr int kTcSingleSetMinRadius = 4;

// Whether a pass of this radius uses the single coefficient set.
inline bool tc_single_set(int radius, bool split_requested) {
    return !split_requested && radius >= kTcSingleSetMinRadius;
}

// True when the device is sm_100 and the shape fits the TMA constraints
// (single-volume passes, radius <= kTcMaxRadiusWide).
bool tc_supported(int radius, int64_t nz, int64_t ny, int64_t nx);

// A field stored with its rows in [y][z][x] order: `base` holds a volume of
// nz_total planes, and a pass works on planes [z0, z0 + nz) of it.
struct YzRows {
    void *base;
    int64_t nz_total, z0;
};

// One z (axis_z) or y pass: out = conv(in) along the axis with a zero
// boundary.  `out` is [z][y][x]; so is `in`, unless in_rows (z pass only)
// gives it in [y][z][x] row order.
template <typename S>
cudaError_t tc_strided(const S *in, S *out, int64_t nz, int64_t ny, int64_t nx, bool axis_z, const float *kernel,
                       int radius, bool error_feedback, cudaStream_t st, const YzRows *in_rows = nullptr,
                       bool hi_only = false);

// The x pass fused with re-illumination; on the last repetition (final_pass)
// it writes the uint16 output and/or the FP32 field (either may be NULL)
// instead of `out`.  out_rows (not final): write the 16-bit field in [y][z][x]
// row order there instead of to `out`.
template <typename S>
cudaError_t tc_contig(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass, uint16_t *out_u16,
                      float *field_out, int64_t nz, int64_t ny, int64_t nx, const float *kernel, int radius,
                      bool error_feedback, cudaStream_t st, const YzRows *out_rows = nullptr, bool hi_only = false);

// True when the fused y + x pass serves the shape (radius <= kTcMaxRadius and
// the tensor-core passes' shape rules).
bool tc_yx_supported(int radius, int64_t nz, int64_t ny, int64_t nx);

// The y and x passes and the re-illumination fused in one kernel per z-plane
// tile: reads the z pass's output `in` ([z][y][x]) and writes the next field
// to `out` ([z][y][x], or [y][z][x] rows at out_rows), or on the last
// repetition (final_pass) the uint16 output and/or the FP32 field.  The fused
// kernel uses one 16-bit coefficient set with the kernel's sum and second
// moment kept (tc_round_taps_matched); hi_only must be true.
template <typename S>
cudaError_t tc_yx(const S *in, S *out, const void *mask, int mask_fmt, bool final_pass, uint16_t *out_u16,
                  float *field_out, int64_t nz, int64_t ny, int64_t nx, const float *kernel, int radius,
                  bool error_feedback, bool hi_only, cudaStream_t st, const YzRows *out_rows = nullptr);

// One 16-bit coefficient per tap of kernel x scale: each tap is one of the two
// representable values around it, chosen (symmetric pairs together) so that
// the rounded kernel's sum and second moment are as close as the format allows
// to the FP32 kernel's.  Plain round-to-nearest changes the sum by ~1e-4, and
// that gain error compounds over the 3 R passes of a diffusion.
void tc_round_taps_matched(const float *kernel, int radius, bool is_bf16, float scale, uint16_t *out);

// tc_round_taps_matched at the scale, among base_scale x (1 + c / C) for 256
// values of c up to radius 32 (32 up to 64, 1 above), whose rounded taps times
// the float 1 / scale the epilogues apply come closest to the FP32 kernel's sum
// (first) and second moment.  A 16-bit grid cannot hit the sum at one scale
// (BF16, sigma 2: 3e-5 off at best), but across scales it comes within 2e-7:
// the gain error that R repetitions compound.  Returns the scale; results are
// cached per kernel.
float tc_round_taps_scaled(const float *kernel, int radius, bool is_bf16, float base_scale, uint16_t *out);

// Reads (and clears) the device error word of the tensor-core kernels:
// 0 = fine, 1..3 = a bounded wait timed out, -1 = could not be read.
int tc_read_and_clear_error();

}  // namespace tc
}  // namespace maxi
