/*
 * CPU restatement of maxibone's mask-diffusion path, used ONLY as test
 * infrastructure: the parity checker for the CUDA library and the timed CPU
 * baseline.  Nothing in the product links or calls this file.
 *
 * Every function restates one function of the reference OpenMP backend
 * (src/lib/cpp/cpu/diffusion.cc) or of the reference bit-packing
 * (src/lib/cpp/cpu_seq/bitpacking.cc), in the same arithmetic order, so that
 * the FP32 results are bit-identical to the reference module built with
 * g++ -O3 on x86-64 (SSE2, no FMA contraction).  The build recipe
 * (oracle/Makefile) passes -ffp-contract=off to keep mul and add separate.
 *
 * Parity pin: tests/test_oracle.py checks this file bit-for-bit against the
 * reference's own `cpu` module compiled from its sources into oracle/_ref
 * (golden vectors in tests/golden/), and against the scipy chain of the
 * reference's own test (src/test/test_diffusion.py:49-59) within 1 LSB.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define MIN(a, b) ((a) < (b) ? (a) : (b))

/* One 1-D convolution along axis `dim` (0=z, 1=y, 2=x) with a zero boundary.
 * Restates cpu_par::diffusion_core, src/lib/cpp/cpu/diffusion.cc:31-57:
 * the tap range is clipped to the volume and the FP32 sum starts at 0 and
 * runs over increasing tap offset r = -min(R, X) .. min(R, N-X-1). */
void oracle_convolve_axis_f32(const float *in, const float *kernel, float *out,
                              int64_t nz, int64_t ny, int64_t nx, int dim, int64_t radius) {
    const int64_t stride[3] = {ny * nx, nx, 1};
    const int64_t ns[3] = {nz, ny, nx};
    #pragma omp parallel for collapse(2) schedule(static)
    for (int64_t i = 0; i < nz; i++) {
        for (int64_t j = 0; j < ny; j++) {
            for (int64_t k = 0; k < nx; k++) {
                const int64_t X[3] = {i, j, k};
                const int64_t lo = -MIN(radius, X[dim]);
                const int64_t hi = MIN(radius, ns[dim] - X[dim] - 1);
                const int64_t o = i * stride[0] + j * stride[1] + k;
                float sum = 0.0f;
                for (int64_t r = lo; r <= hi; r++) {
                    float prod = in[o + r * stride[dim]] * kernel[radius + r];
                    sum = sum + prod;
                }
                out[o] = sum;
            }
        }
    }
}

/* FP64 version of the same convolution, used as the error reference for the
 * reduced-precision field forms. */
void oracle_convolve_axis_f64(const double *in, const double *kernel, double *out,
                              int64_t nz, int64_t ny, int64_t nx, int dim, int64_t radius) {
    const int64_t stride[3] = {ny * nx, nx, 1};
    const int64_t ns[3] = {nz, ny, nx};
    #pragma omp parallel for collapse(2) schedule(static)
    for (int64_t i = 0; i < nz; i++) {
        for (int64_t j = 0; j < ny; j++) {
            for (int64_t k = 0; k < nx; k++) {
                const int64_t X[3] = {i, j, k};
                const int64_t lo = -MIN(radius, X[dim]);
                const int64_t hi = MIN(radius, ns[dim] - X[dim] - 1);
                const int64_t o = i * stride[0] + j * stride[1] + k;
                double sum = 0.0;
                for (int64_t r = lo; r <= hi; r++) sum += in[o + r * stride[dim]] * kernel[radius + r];
                out[o] = sum;
            }
        }
    }
}

/* u8 mask -> {0,1} field.  Restates convert_uint8_to_float,
 * src/lib/cpp/cpu/diffusion.cc:243-247 (`src > 0 ? 1 : 0`). */
void oracle_u8_to_f32(const uint8_t *src, float *dst, int64_t n) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) dst[i] = src[i] > 0 ? 1.0f : 0.0f;
}

/* Re-illumination.  Restates illuminate, src/lib/cpp/cpu/diffusion.cc:295-302. */
void oracle_illuminate_f32(const uint8_t *mask, float *field, int64_t n) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) if (mask[i] > 0) field[i] = 1.0f;
}

/* Quantisation.  Restates convert_float_to_uint16,
 * src/lib/cpp/cpu/diffusion.cc:191-195: (uint16_t) floor(v * 65535.0f) in FP32. */
void oracle_f32_to_u16(const float *src, uint16_t *dst, int64_t n) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) dst[i] = (uint16_t) floorf(src[i] * 65535.0f);
}

/* The in-memory driver.  Restates diffusion_in_memory and diffusion_step,
 * src/lib/cpp/cpu/diffusion.cc:339-374 and :314-320: u8 -> f32, then for each
 * repetition the z, y, x passes with ping-pong buffers followed by
 * illumination, then f32 -> u16.  `field_out` (may be NULL) receives the final
 * FP32 field, which the reference keeps internal.  Returns 0, or -1 when the
 * working buffers cannot be allocated. */
int oracle_diffusion_in_memory(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                               const float *kernel, int64_t kernel_size, int64_t repititions,
                               uint16_t *output, float *field_out) {
    const int64_t n = nz * ny * nx, radius = kernel_size / 2;
    float *b0 = (float *) malloc((size_t) n * sizeof(float));
    float *b1 = (float *) malloc((size_t) n * sizeof(float));
    if (!b0 || !b1) { free(b0); free(b1); return -1; }
    oracle_u8_to_f32(voxels, b0, n);
    for (int64_t rep = 0; rep < repititions; rep++) {
        for (int dim = 0; dim < 3; dim++) {
            oracle_convolve_axis_f32(b0, kernel, b1, nz, ny, nx, dim, radius);
            float *t = b0; b0 = b1; b1 = t;
        }
        oracle_illuminate_f32(voxels, b0, n);
    }
    if (output) oracle_f32_to_u16(b0, output, n);
    if (field_out) memcpy(field_out, b0, (size_t) n * sizeof(float));
    free(b0);
    free(b1);
    return 0;
}

/* The same driver in FP64 throughout (kernel given in FP64).  This is the
 * error reference for the BF16/FP16 field forms; it has no reference
 * counterpart beyond the algorithm above.  Returns 0 or -1 on allocation failure. */
int oracle_diffusion_f64(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                         const double *kernel, int64_t kernel_size, int64_t repititions,
                         double *field_out) {
    const int64_t n = nz * ny * nx, radius = kernel_size / 2;
    double *b0 = (double *) malloc((size_t) n * sizeof(double));
    double *b1 = (double *) malloc((size_t) n * sizeof(double));
    if (!b0 || !b1) { free(b0); free(b1); return -1; }
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) b0[i] = voxels[i] > 0 ? 1.0 : 0.0;
    for (int64_t rep = 0; rep < repititions; rep++) {
        for (int dim = 0; dim < 3; dim++) {
            oracle_convolve_axis_f64(b0, kernel, b1, nz, ny, nx, dim, radius);
            double *t = b0; b0 = b1; b1 = t;
        }
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) if (voxels[i] > 0) b0[i] = 1.0;
    }
    memcpy(field_out, b0, (size_t) n * sizeof(double));
    free(b0);
    free(b1);
    return 0;
}

/* One repetition of the on-disk variant's semantics on an in-memory field:
 * the mask is rebuilt from the field as `field == 1.0f` before the step.
 * Restates store_mask (src/lib/cpp/cpu/diffusion.cc:304-312) followed by
 * diffusion_step (:314-320) as used by diffusion_on_disk (:420-421), and the
 * GPU backend's final uint16 conversion (src/lib/cpp/gpu/diffusion.cc:937).
 * The slab decomposition of the reference is exact for the z-pass of the core
 * layers (radius-layer halos), so the whole-volume form gives the same values. */
int oracle_diffusion_on_disk_field(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                                   const float *kernel, int64_t kernel_size, int64_t repititions,
                                   float *field_out) {
    const int64_t n = nz * ny * nx, radius = kernel_size / 2;
    float *b0 = (float *) malloc((size_t) n * sizeof(float));
    float *b1 = (float *) malloc((size_t) n * sizeof(float));
    uint8_t *mask = (uint8_t *) malloc((size_t) n);
    if (!b0 || !b1 || !mask) { free(b0); free(b1); free(mask); return -1; }
    oracle_u8_to_f32(voxels, b0, n);
    for (int64_t rep = 0; rep < repititions; rep++) {
        #pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; i++) mask[i] = b0[i] == 1.0f ? 1 : 0;
        for (int dim = 0; dim < 3; dim++) {
            oracle_convolve_axis_f32(b0, kernel, b1, nz, ny, nx, dim, radius);
            float *t = b0; b0 = b1; b1 = t;
        }
        oracle_illuminate_f32(mask, b0, n);
    }
    memcpy(field_out, b0, (size_t) n * sizeof(float));
    free(b0);
    free(b1);
    free(mask);
    return 0;
}

int oracle_diffusion_on_disk_semantics(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                                       const float *kernel, int64_t kernel_size, int64_t repititions,
                                       uint16_t *output) {
    const int64_t n = nz * ny * nx;
    float *f = (float *) malloc((size_t) n * sizeof(float));
    if (!f) return -1;
    const int rc = oracle_diffusion_on_disk_field(voxels, nz, ny, nx, kernel, kernel_size, repititions, f);
    if (rc == 0) oracle_f32_to_u16(f, output, n);
    free(f);
    return rc;
}

/* Repetitions continued from a given FP32 field (the field after earlier
 * repetitions) on a sub-volume whose first / last planes may be halo planes:
 * the same steps as oracle_diffusion_in_memory (conv z, y, x with a zero
 * boundary at the sub-volume's edges, illuminate) without the initial
 * mask -> field conversion.  Planes at least reps x radius from a cut edge
 * hold the whole volume's values afterwards. */
int oracle_diffusion_from_field(const float *field_in, const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                                const float *kernel, int64_t kernel_size, int64_t repititions, float *field_out) {
    const int64_t n = nz * ny * nx, radius = kernel_size / 2;
    float *b0 = (float *) malloc((size_t) n * sizeof(float));
    float *b1 = (float *) malloc((size_t) n * sizeof(float));
    if (!b0 || !b1) { free(b0); free(b1); return -1; }
    memcpy(b0, field_in, (size_t) n * sizeof(float));
    for (int64_t rep = 0; rep < repititions; rep++) {
        for (int dim = 0; dim < 3; dim++) {
            oracle_convolve_axis_f32(b0, kernel, b1, nz, ny, nx, dim, radius);
            float *t = b0; b0 = b1; b1 = t;
        }
        oracle_illuminate_f32(voxels, b0, n);
    }
    memcpy(field_out, b0, (size_t) n * sizeof(float));
    free(b0);
    free(b1);
    return 0;
}

/* The CPU backend's final conversion of its on-disk variant,
 * convert_float_to_uint8 (src/lib/cpp/cpu/diffusion.cc:139-144):
 * (uint8_t) floor(v * 255.0f) in FP32. */
void oracle_f32_to_u8(const float *field, uint8_t *out, int64_t n) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i++) out[i] = (uint8_t) floorf(field[i] * 255.0f);
}

/* Bit-packing, uint32 words, most significant bit first.  Restates
 * cpu_seq::encode / decode, src/lib/cpp/cpu_seq/bitpacking.cc:9-42
 * (`(mask[i+j] & 1) << (31-j)`).  n must be a multiple of 32. */
void oracle_bitpack_encode_u32(const uint8_t *mask, int64_t n, uint32_t *packed) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i += 32) {
        uint32_t w = 0;
        for (int j = 0; j < 32; j++) w |= (uint32_t) (mask[i + j] & 1) << (31 - j);
        packed[i / 32] = w;
    }
}

void oracle_bitpack_decode_u32(const uint32_t *packed, int64_t n, uint8_t *mask) {
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; i += 32) {
        uint32_t w = packed[i / 32];
        for (int j = 0; j < 32; j++) mask[i + j] = (uint8_t) ((w >> (31 - j)) & 1);
    }
}
