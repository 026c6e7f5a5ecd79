/*
 * maxibone_diffusion.h -- C ABI of the B200 (sm_100a) mask-diffusion library.
 *
 * The path: a uint8 binary mask becomes a {0,1} field; each repetition applies
 * a 1-D kernel along z, then y, then x with a zero boundary, and re-illuminates
 * the mask voxels to exactly 1.0; the final field is quantised to uint16 as
 * floor(v * 65535) in FP32.  All entry points return a maxi_status; a nonzero
 * code comes with a message from maxi_last_error() (per calling thread).
 *
 * Plain C types only: pointers, sizes, enums.  No ownership crosses the
 * boundary; the caller owns every buffer it passes in.  Calls are synchronous
 * unless the entry point takes a `stream` (a cudaStream_t; NULL = the legacy
 * default stream), in which case work is enqueued on that stream.
 */
#ifndef MAXIBONE_DIFFUSION_H
#define MAXIBONE_DIFFUSION_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum maxi_status {
    MAXI_OK = 0,
    MAXI_ERR_INVALID_ARGUMENT = 1, /* bad shape, kernel length, dtype, pointer */
    MAXI_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    MAXI_ERR_OUT_OF_MEMORY = 3,    /* device or pinned host allocation failed */
    MAXI_ERR_IO = 4,               /* file open / read / write failed (on-disk form) */
    MAXI_ERR_UNSUPPORTED = 5,      /* a valid request this library does not serve */
    MAXI_ERR_NO_DEVICE = 6         /* no CUDA device visible */
} maxi_status;

/* How the field is stored in HBM between passes.  Accumulation is always FP32
 * (FP64 for MAXI_FIELD_F64). */
typedef enum maxi_field_type {
    MAXI_FIELD_F32 = 0,
    MAXI_FIELD_BF16 = 1,
    MAXI_FIELD_F16 = 2,
    MAXI_FIELD_F64 = 3 /* FP64 storage and arithmetic: the error reference form */
} maxi_field_type;

/* Mask encodings accepted by the device entry points. */
typedef enum maxi_mask_format {
    MAXI_MASK_U8 = 0,       /* one byte per voxel, voxel is set when > 0 */
    MAXI_MASK_BITPACKED = 1 /* uint32 words over the flat voxel order, 32 voxels each,
                               most significant bit first (the reference bitpacking
                               layout); ceil(nz*ny*nx / 32) words */
} maxi_mask_format;

/* Option bits for maxi_diffusion_device(). */
#define MAXI_FLAG_REFERENCE_ROUNDING 0x1 /* FP32 only: separate multiply and add in the
                                            reference's tap order, bit-identical to the
                                            reference OpenMP backend */
#define MAXI_FLAG_NO_TENSOR_CORES 0x2    /* BF16/FP16: CUDA-core passes only */
#define MAXI_FLAG_MASK_FROM_FIELD 0x8    /* FP32 only: before every repetition after the first,
                                            the mask is rebuilt as `field == 1.0f` -- the
                                            semantics of the reference's on-disk variant */
#define MAXI_FLAG_AUTOTUNE 0x10          /* batch plans: time each tensor-core group's forms
                                            (one batched launch per pass, per-volume tensor-core
                                            launches, per-volume CUDA-core passes) and keep the
                                            fastest (cached per process and in a JSON file) */
#define MAXI_FLAG_NEAREST_ROUNDING 0x4   /* BF16/FP16: plain round-to-nearest stores instead of
                                            error-feedback rounding along x (the default for
                                            radius >= 4, which keeps the stored rounding noise
                                            out of the result) */
#define MAXI_FLAG_SEPARATE_PASSES 0x20   /* BF16/FP16 tensor cores: the y and x passes as two
                                            kernels (two HBM round trips) instead of the fused
                                            y + x kernel, which is the default where it applies
                                            (radius 4 to 32: the single coefficient set) */
#define MAXI_FLAG_SPLIT_COEFFICIENTS 0x40 /* BF16/FP16 tensor cores: Toeplitz coefficients as high +
                                            low 16-bit halves (two MMAs per K step) instead of the
                                            single set whose taps are rounded so that the
                                            kernel's sum and second moment are kept (the default
                                            from radius 4; smaller radii always use the halves);
                                            runs the separate y and x passes */

const char *maxi_last_error(void);
const char *maxi_version(void);

/* Kernel families a diffusion call enqueued (bits of maxi_last_path()). */
#define MAXI_PATH_CUDA_CORES 0x1         /* unrolled CUDA-core passes (any of z, y, x) */
#define MAXI_PATH_TENSOR_CORES_ZY 0x2    /* tcgen05 z and y passes */
#define MAXI_PATH_TENSOR_CORES_X 0x4     /* tcgen05 x pass + re-illumination */
#define MAXI_PATH_FUSED_YX 0x8           /* tcgen05 y and x passes fused in one kernel */
#define MAXI_PATH_GENERIC 0x10           /* generic passes: FP64, reference rounding, radius > 128 */
#define MAXI_PATH_FP32_FALLBACK 0x20     /* a 16-bit field was requested on a shape the tensor-core
                                            passes do not take; the FP32 form ran instead */

/*
 * MAXI_PATH_* bits of the last maxi_diffusion_device() call made by this
 * thread (no reference counterpart: the reference has one code path per
 * build).  Lets callers and tests see which kernels served a request, e.g.
 * that a BF16 request ran on the tensor cores and not on a fallback.
 */
int maxi_last_path(void);

/*
 * Status of the tensor-core passes since the last call: their waits are
 * bounded (about one second); a pass that gave up records a code here instead
 * of hanging.  Synchronises with the device; returns MAXI_OK or MAXI_ERR_CUDA
 * (message from maxi_last_error()) and clears the recorded code.
 */
int maxi_tensor_core_status(void);

/*
 * The single 16-bit coefficient set the tensor-core passes use for this
 * kernel (no counterpart in the reference, whose passes use the FP32 kernel;
 * for inspection and tests): taps[kernel_size] receives the BF16 or FP16 bit
 * patterns (field_type MAXI_FIELD_BF16 / MAXI_FIELD_F16) and *inv_scale the
 * factor the passes' epilogues apply to the accumulated sums, so that the
 * pass computes sum_i from16(taps[i]) * inv_scale * field.  kernel_size odd,
 * at most 257.
 */
int maxi_tensor_core_taps(const float *kernel, int64_t kernel_size, int32_t field_type, uint16_t *taps,
                          float *inv_scale);

/* Kernel kinds reported by maxi_profile_read(). */
typedef enum maxi_kernel_kind {
    MAXI_KERNEL_INIT = 0,    /* mask -> field */
    MAXI_KERNEL_Z = 1,       /* z pass */
    MAXI_KERNEL_Y = 2,       /* y pass */
    MAXI_KERNEL_X = 3,       /* x pass + re-illumination */
    MAXI_KERNEL_X_FINAL = 4, /* last x pass + re-illumination + uint16 quantisation */
    MAXI_KERNEL_YX = 5,      /* fused y and x passes + re-illumination */
    MAXI_KERNEL_OTHER = 6,
    MAXI_KERNEL_KINDS = 8
} maxi_kernel_kind;

/*
 * Per-launch timing of this library's kernels (no reference counterpart; the
 * reference times slabs with wall clocks behind a PROFILE constant,
 * src/lib/cpp/gpu/diffusion.cc:854-933).  When enabled, every kernel launch is
 * bracketed by CUDA events on its stream.  maxi_profile_read() waits for the
 * recorded events, writes the summed device milliseconds and launch counts per
 * maxi_kernel_kind (n_kinds entries) and clears the record.
 */
int maxi_profile_enable(int on);
int maxi_profile_read(double *ms_by_kind, int64_t *launches_by_kind, int32_t n_kinds);

/*
 * In-memory diffusion on HOST buffers (the reference-facing call).
 * Replaces NS::diffusion_in_memory, src/lib/cpp/include/diffusion.hh:36, as
 * bound by python_api::diffusion_in_memory, src/pybind/diffusion-pybind.cc:27-53.
 * voxels: uint8[nz][ny][nx] (set when > 0); kernel: float[kernel_size], odd
 * length; output: uint16[nz][ny][nx], written in place.  FP32 field.
 * Pageable (not pinned) buffers of 64 MiB or more cross through two 32 MiB
 * pinned staging buffers allocated for the call, several host threads moving
 * each chunk while the previous one crosses PCIe; pinned buffers are copied
 * directly.
 */
int maxi_diffusion_in_memory(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                             const float *kernel, int64_t kernel_size, int64_t repititions,
                             uint16_t *output, int verbose);

/*
 * maxi_diffusion_in_memory() allocates its device buffers per call and frees
 * them before it returns, as the reference does (src/lib/cpp/cpu/diffusion.cc:
 * 343-345,371-373).  maxi_keep_device_buffers(1) makes it keep them between
 * calls instead (one grow-only allocation per device), so repeated calls do
 * not map gigabytes each time; maxi_keep_device_buffers(0) restores the
 * default and frees them, as does maxi_release_cached_memory() (which also
 * frees the sphere-morphology scratch).  Volumes larger than the device go to
 * the out-of-core form, as the reference's pybind module does
 * (src/pybind/diffusion-pybind.cc:40-45).
 */
int maxi_keep_device_buffers(int keep);
int maxi_release_cached_memory(void);

/*
 * Working memory (bytes) that maxi_diffusion_device() needs for one volume:
 * two field buffers of the storage type plus the bit-packed mask.
 */
int64_t maxi_diffusion_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t field_type);

/*
 * In-memory diffusion on DEVICE buffers, enqueued on `stream`.  The device
 * form of diffusion.hh:36 (no reference counterpart for the extra options).
 *   mask: device mask in `mask_format`;
 *   kernel: HOST float[kernel_size] (copied into the launch parameters);
 *   output: device uint16[nz][ny][nx], or NULL;
 *   field_out: device buffer for the final field before quantisation, or NULL:
 *              float[N] for F32/BF16/F16 (taken from the FP32 accumulator),
 *              double[N] for F64;
 *   workspace: device memory of at least maxi_diffusion_workspace_size() bytes,
 *              256-byte aligned, or NULL to let the library allocate (and
 *              free) it per call;  a bit-packed mask must be 4-byte aligned
 *              (misaligned pointers are rejected with MAXI_ERR_INVALID_ARGUMENT);
 *   flags: MAXI_FLAG_* bits.
 */
int maxi_diffusion_device(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                          const float *kernel, int64_t kernel_size, int64_t repititions,
                          uint16_t *output, void *field_out, int32_t field_type, int32_t flags,
                          void *workspace, int64_t workspace_bytes, void *stream);

/*
 * maxi_diffusion_device() for one z-slab of a volume split over several GPUs
 * or processed in rounds (no reference counterpart; the reference's blocks
 * exchange halos through host memory every repetition,
 * src/lib/cpp/gpu/diffusion.cc:1013-1073).
 *   init_field: device FP32 field of the slab's nz planes to start from
 *               (the field after earlier repetitions), or NULL to start from
 *               the mask as maxi_diffusion_device() does;
 *   shrink_lo / shrink_hi: repetition k runs only on planes
 *               [k * shrink_lo, nz - k * shrink_hi) -- the planes that can still
 *               reach the slab's core when the slab's first / last planes are
 *               halo planes of a cut, not the volume's edge (pass the radius
 *               there, else 0); shrinking needs (ny * nx) % 32 == 0 and the
 *               unrolled passes (else the whole slab is computed, also exact).
 *               With shrinking, the last repetition writes output / field_out
 *               only on planes [(R-1) * shrink_lo, nz - (R-1) * shrink_hi).
 * After R repetitions the planes at least R x radius from every cut side hold
 * the whole volume's values.  The rebuilt-mask flag (MAXI_FLAG_MASK_FROM_FIELD)
 * rebuilds the mask from init_field before the first repetition as well.
 */
int maxi_diffusion_device_ex(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                             const float *kernel, int64_t kernel_size, int64_t repititions, uint16_t *output,
                             void *field_out, int32_t field_type, int32_t flags, void *workspace,
                             int64_t workspace_bytes, void *stream, const float *init_field, int64_t shrink_lo,
                             int64_t shrink_hi);

/*
 * Allocation-free variant of maxi_diffusion_device() for the FP32 field.  It
 * has no counterpart in the reference.  It serves callers that may not
 * allocate device memory while they run (a host that owns the whole device
 * heap through its own sub-allocator, a fixed memory budget set at start-up,
 * code that cannot accept an allocation's synchronisation or failure in the
 * middle of its work): the two field buffers come from a fixed 64 MiB array
 * inside the library, so no cudaMalloc or other allocation happens.
 *   - at most 8,388,608 voxels (2^23) per call, radius <= 128, repititions >= 1;
 *     anything larger is rejected with MAXI_ERR_INVALID_ARGUMENT (radius:
 *     MAXI_ERR_UNSUPPORTED) before GPU work starts;
 *   - the array stays reserved until the process exits on each GPU where the
 *     library's device code is loaded: with CUDA's default lazy module loading
 *     the GPUs that use this call, with CUDA_MODULE_LOADING=EAGER every GPU the
 *     process creates a context on; the first call on a device looks up its
 *     address (cudaGetSymbolAddress), so make that first call before any
 *     stream capture;
 *   - all calls share the array: calls whose GPU work overlaps (different
 *     streams or threads without ordering) race and give wrong results.
 * mask, output (uint16, or NULL) and field_out (float, or NULL) are device
 * buffers supplied by the caller; work is enqueued on `stream`.
 */
int maxi_diffusion_device_noalloc(const void *mask, int32_t mask_format, int64_t nz, int64_t ny, int64_t nx,
                                  const float *kernel, int64_t kernel_size, int64_t repititions,
                                  uint16_t *output, float *field_out, void *stream);

/*
 * Batched form (no reference counterpart: the reference diffuses one volume
 * per call).  Many independent DEVICE volumes of uneven sizes, each with its
 * own kernel and repetition count, run as one CUDA graph; on the tensor-core
 * path every pass of every repetition is one persistent launch over the tiles
 * of all volumes that share a kernel and a repetition count.
 */
typedef struct maxi_volume {
    const void *mask;      /* device uint8 [nz][ny][nx], set when > 0 */
    uint16_t *output;      /* device uint16 [nz][ny][nx], or NULL */
    float *field_out;      /* device float [nz][ny][nx] final field, or NULL */
    int64_t nz, ny, nx;
    const float *kernel;   /* host float[kernel_size], odd length, radius <= 128 (copied) */
    int64_t kernel_size;
    int64_t repititions;   /* >= 1 */
} maxi_volume;

typedef struct maxi_batch_plan maxi_batch_plan; /* opaque */

/* Allocates the workspace of all volumes, groups them, optionally autotunes
 * (MAXI_FLAG_AUTOTUNE, timing on `stream`) and captures the repetition loop
 * into a CUDA graph.  Field types F32, BF16, F16.
 * Tuning choices are keyed by GPU name and SM count, field type, radius and the
 * group's volume shapes, and persisted in the JSON file named by the
 * environment variable MAXIBONE_TUNE_CACHE (an empty value: no file), else
 * $XDG_CACHE_HOME/maxibone_b200/batch_tune.json or
 * ~/.cache/maxibone_b200/batch_tune.json. */
int maxi_batch_plan_create(const maxi_volume *volumes, int64_t n_volumes, int32_t field_type, int32_t flags,
                           void *stream, maxi_batch_plan **plan);
/* Launches the plan's graph on `stream` (asynchronous; may be replayed). */
int maxi_batch_plan_run(maxi_batch_plan *plan, void *stream);
/* Text summary of the plan's groups and tuning decisions. */
int maxi_batch_plan_describe(const maxi_batch_plan *plan, char *buffer, int64_t buffer_bytes);
/* Waits for the device and frees the plan. */
int maxi_batch_plan_destroy(maxi_batch_plan *plan);
/* Drops the process's tuning choices: the next autotuned plan reads the cache
 * file again (and times what it does not hold). */
int maxi_batch_tune_forget(void);
/* create + run + synchronise + destroy. */
int maxi_diffusion_batched(const maxi_volume *volumes, int64_t n_volumes, int32_t field_type, int32_t flags,
                           void *stream);

/*
 * Out-of-core diffusion of a HOST volume that need not fit the device.
 * Replaces NS::diffusion_out_of_core, src/lib/cpp/include/diffusion.hh:74
 * (GPU body src/lib/cpp/gpu/diffusion.cc:947-1129).  The volume is processed as
 * z-slabs of at most global_z planes (thinner when such slabs do not fit the
 * device) that span the full y and x extent (global_y / global_x only have to
 * be positive).  Each slab is loaded with repititions x radius halo planes per
 * side so all repetitions run on the device without exchanges; when such halos
 * leave no room for useful slabs (large repititions x radius), the repetitions
 * run in rounds of k with k x radius halos and the field goes through host
 * memory between rounds (8 bytes per voxel of pinned host memory; only when
 * that fits half of the host's available memory, MemAvailable, or
 * MAXIBONE_OOC_HOST_BUDGET bytes when that environment variable is set).  Planes of
 * a multiple of 32 voxels keep the whole mask bit-packed on the device; from a
 * pinned `voxels` buffer it is uploaded in chunks of about 1 GiB
 * (MAXIBONE_OOC_UPLOAD_CHUNK_PLANES planes when set) while the first slabs run.
 * FP32 field; results equal maxi_diffusion_in_memory().
 */
int maxi_diffusion_out_of_core(const uint8_t *voxels, int64_t total_z, int64_t total_y, int64_t total_x,
                               int64_t global_z, int64_t global_y, int64_t global_x, const float *kernel,
                               int64_t kernel_size, int64_t repititions, uint16_t *output, int verbose);

/* The same with the field storage type and MAXI_FLAG_* options; slab_z = 0
 * lets the library choose the slab depth. */
int maxi_diffusion_out_of_core_ex(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx, int64_t slab_z,
                                  const float *kernel, int64_t kernel_size, int64_t repititions, uint16_t *output,
                                  int32_t field_type, int32_t flags, int verbose);

/*
 * The out-of-core plan maxi_diffusion_out_of_core_ex() would use (no
 * reference counterpart: the reference's block size is fixed by the caller).
 * For `device_bytes` of free device memory (0: the current device's free
 * memory, or MAXIBONE_OOC_DEVICE_BUDGET bytes when that environment variable
 * is set and smaller) writes the slab depth, the repetitions per round (equal
 * to repititions: one round with deep halos, no exchange) and whether the mask
 * stays bit-packed on the device.  Exchange rounds are only planned when their
 * 8 bytes per voxel fit the host memory that may be pinned (see
 * maxi_diffusion_out_of_core).  MAXI_ERR_OUT_OF_MEMORY when no slab fits.
 */
int maxi_out_of_core_plan(int64_t nz, int64_t ny, int64_t nx, int64_t slab_z, int64_t kernel_size,
                          int64_t repititions, int32_t field_type, int32_t flags, int64_t device_bytes,
                          int64_t *slab_planes, int64_t *reps_per_round, int32_t *resident_mask);

/*
 * On-disk diffusion: raw uint8 volume file in, raw uint16 file out.  Replaces
 * NS::diffusion_on_disk, src/lib/cpp/include/diffusion.hh:55, as bound by
 * python_api::diffusion_on_disk, src/pybind/diffusion-pybind.cc:67-77 (GPU
 * semantics: uint16 output, src/lib/cpp/gpu/diffusion.cc:937; the mask of each
 * repetition is rebuilt as field == 1.0f).  Streams z-slabs of global_z planes;
 * writes no temporary files.
 */
int maxi_diffusion_on_disk(const char *input_file, const float *kernel, int64_t kernel_size, const char *output_file,
                           int64_t total_z, int64_t total_y, int64_t total_x, int64_t global_z, int64_t global_y,
                           int64_t global_x, int64_t repititions, int verbose);

/*
 * Bit-packing of a device mask to uint32 words, MSB first.  Replaces the
 * reference `bitpacking.encode` / `decode` (src/pybind/bitpacking-pybind.cc:17-48,
 * src/lib/cpp/cpu_seq/bitpacking.cc:9-42); n must be a multiple of 32.
 * encode keeps bit 0 of each byte (`mask & 1`), as the reference does.
 */
int maxi_bitpack_encode(const uint8_t *mask, int64_t n, uint32_t *packed, void *stream);
int maxi_bitpack_decode(const uint32_t *packed, int64_t n, uint8_t *mask, void *stream);

/*
 * Combination of the Gaussian (diffusion) field and the implant EDT field into
 * one uint16 field: the step after the diffusion in maxibone's pipeline
 * (src/processing_steps/0975_combine_fields.py:38-62, with its to_int from
 * src/lib/cpp/include/general.hh:78-118), bit-identical to it.  gauss, edt,
 * output: device uint16[nz][ny][nx]; the cylinder mask spans y and x as
 * generate_cylinder_mask(ny, nx) (the script's generate_cylinder_mask(nx) for
 * square planes).  Three passes over both fields with two small read-backs, so
 * the call synchronises the stream.  A field whose maximum is 0 is rejected
 * (the reference divides by it).
 */
int maxi_combine_fields(const uint16_t *gauss, const uint16_t *edt, int64_t nz, int64_t ny, int64_t nx,
                        uint16_t *output, void *stream);

/*
 * The implant cylinder mask applied to a uint16 field in place: voxels outside
 * generate_cylinder_mask(ny, nx) (src/lib/py/helpers.py:411-434; the reference
 * calls it with nx for its square planes) become 0, as the diffusion step's
 * `result * cylinder_mask` before saving (src/processing_steps/
 * 0900_generate_gauss_c.py:117,124).  Only the outside voxels are written.
 * field: device uint16[nz][ny][nx].  Synchronises the stream.
 */
int maxi_mask_cylinder(uint16_t *field, int64_t nz, int64_t ny, int64_t nx, void *stream);

/*
 * 3-D sphere dilation (dilate != 0) or erosion of a mask: the reference's morphology
 * module (src/lib/cpp/cpu_seq/morphology.cc:14-99 and gpu/morphology.cc:14-101, bound
 * as dilate_3d_sphere / erode_3d_sphere by src/pybind/morphology-pybind.cc:24-45,
 * 147,149).  voxels, result: device uint8[nz][ny][nx]; result[z,y,x] = 1 iff some
 * in-volume voxel within the sphere (pz^2 + py^2 + px^2 <= radius^2) is nonzero
 * (dilation) / every one has bit 0 set (erosion), else 0.  radius <= 32 (larger
 * spheres: repeated calls, as the reference's morph_3d does with radius 16).
 * Synchronises the stream.
 */
int maxi_morphology_sphere(const uint8_t *voxels, uint8_t *result, int64_t nz, int64_t ny, int64_t nx,
                           int64_t radius, int dilate, void *stream);

/*
 * The same on a bit-packed mask: dilate_3d_sphere_bitpacked / erode_3d_sphere_bitpacked
 * (src/lib/cpp/gpu/morphology.cc:103-176, src/pybind/morphology-pybind.cc:61-77,148,150).
 * voxels, result: device uint32[nz][ny][nw], 32 voxels per word, MSB first along x.
 * With the reference GPU build's shifts (by 32 or more, or by a negative amount: 0)
 * its per-(pz, py) kernel rows hold x offsets -radius .. 31 - radius, so the sphere
 * is clipped at x offset 31 - radius; this entry point computes exactly that.
 * radius <= 31.  Synchronises the stream.
 */
int maxi_morphology_sphere_bitpacked(const uint32_t *voxels, uint32_t *result, int64_t nz, int64_t ny,
                                     int64_t nw, int64_t radius, int dilate, void *stream);

/*
 * The implant's front / back / shell / solid masks in its frame of reference: the
 * reference's compute_front_back_masks (src/lib/cpp/cpu_seq/geometry.cc:112-215,
 * bound by src/pybind/geometry-pybind.cc:283-310), run by
 * src/processing_steps/0750_bone_region.py:62 to make the implant_solid mask the
 * diffusion step diffuses.  mask and the four outputs: device uint8[nz][ny][nx];
 * E, cm, cp, UVWp: HOST float arrays of 9, 3, 3 and 9 values (row-major 3x3).
 * Identical to the reference (FP32 in its operation order, no fused multiply-add;
 * the 0.7 * rmax comparisons in FP64).  Axes up to 2^24.  Synchronises the stream.
 */
int maxi_implant_masks(const uint8_t *mask, int64_t nz, int64_t ny, int64_t nx, float voxel_size, const float *E,
                       const float *cm, const float *cp, const float *UVWp, uint8_t *front_mask, uint8_t *back_mask,
                       uint8_t *implant_shell_mask, uint8_t *solid_implant, void *stream);

/*
 * 2-D histogram of (field value, voxel value) pairs, added into bins: the
 * reference's field_histogram (src/lib/cpp/cpu/histograms.cc:231-305, bound by
 * src/pybind/histograms-pybind.cc:81-107), the consumer of the diffusion field
 * (src/processing_steps/1000_compute_histograms.py:80-115).  voxels: device
 * uint16[nZ][nY][nX]; field: device uint16[nz][ny][nx], read at
 * (min(nz-1, floor(Z*nz/nZ)), floor(Y*ny/nY), floor(X*nx/nX)); bins: device
 * uint64[field_bins][voxel_bins], accumulated into (not cleared).  Rows start at
 * y_start and columns at x_start (the offset's y and x; its z is unused, as in
 * the reference).  Voxel values outside [vmin, vmax], zero voxels and zero field
 * values are skipped; bin indices use the reference's FP64 expressions, so the
 * counts are identical.  Field values whose bin falls outside [0, field_bins)
 * are skipped (the reference writes out of bounds there).  Synchronises the stream.
 */
int maxi_field_histogram(const uint16_t *voxels, int64_t nZ, int64_t nY, int64_t nX, const uint16_t *field,
                         int64_t nz, int64_t ny, int64_t nx, int64_t y_start, int64_t x_start, uint64_t *bins,
                         int64_t field_bins, int64_t voxel_bins, double vmin, double vmax, double fmin, double fmax,
                         void *stream);

/*
 * Per-axis and radial histograms of a z-block of a volume, added into the bins:
 * the reference's axis_histograms (src/lib/cpp/cpu/histograms.cc:14-80, bound by
 * src/pybind/histograms-pybind.cc:30-66; called per block by
 * src/processing_steps/1000_compute_histograms.py:470).  voxels: device
 * uint16[nz_block][Ny][Nx] holding global planes z_start .. z_start + nz_block
 * (planes at or past Nz are ignored); x_bins [Nx][voxel_bins], y_bins
 * [Ny][voxel_bins], z_bins [Nz][voxel_bins], r_bins [n_r][voxel_bins]: device
 * uint64, accumulated into.  Each voxel at y >= y_start, x >= x_start whose value
 * lies in [vmin, vmax] and is nonzero is binned as
 * floor((voxel_bins - 1) * ((v - vmin) / (vmax - vmin))) (FP64) and counted in
 * row x, y, z and floor(sqrt((x-cx)^2 + (y-cy)^2)) of the four histograms;
 * radii at or past n_r (out-of-bounds writes in the reference) are skipped.
 * Counts are identical to the reference's.  Synchronises the stream.
 */
int maxi_axis_histograms(const uint16_t *voxels, int64_t nz_block, int64_t Nz, int64_t Ny, int64_t Nx,
                         int64_t z_start, int64_t y_start, int64_t x_start, uint64_t *x_bins, uint64_t *y_bins,
                         uint64_t *z_bins, uint64_t *r_bins, int64_t voxel_bins, int64_t n_r, int64_t cy, int64_t cx,
                         double vmin, double vmax, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* MAXIBONE_DIFFUSION_H */
