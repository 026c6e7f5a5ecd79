// Out-of-core diffusion: volumes held in host memory (or files) that do not
// fit the device, processed as z-slabs with deep halos.
//
// The reference's out-of-core form (src/lib/cpp/gpu/diffusion.cc:947-1129)
// cuts the volume into 3-D blocks with a radius halo and exchanges halos
// through host memory on every repetition.  Here each z-slab of S planes is
// loaded once with H = repetitions x radius extra planes on each side, all
// repetitions run on the device, and only the slab's own S planes are written
// back: a voxel's value after R repetitions depends only on input planes
// within R x radius of it (one z pass per repetition), so the core planes are
// exact and no exchange between slabs is needed.  The halo's width is only
// needed at the first repetition: repetition k runs on the planes that are at
// least k x radius from a cut side, which brings the computed planes per slab
// from R x (S + 2H) down to about R x (S + H).  Two slab contexts on
// separate streams overlap one slab's host<->device copies with the other's
// compute; pageable host buffers are staged through pinned memory by the host
// thread while the device works.
#include <cstdio>
#include <cstring>
#include <vector>
#include <functional>

#include "host_util.h"
#include "unrolled.h"

namespace maxi {

struct OocContext {
    cudaStream_t stream = nullptr;
    uint8_t *d_mask = nullptr;
    uint16_t *d_out = nullptr;
    void *ws = nullptr;
    int64_t ws_bytes = 0;
    uint8_t *h_in = nullptr;    // pinned staging (pageable input only)
    uint16_t *h_out = nullptr;  // pinned staging (pageable output only)
    // pending copy-out of the slab this context last processed
    bool pending = false;
    int64_t out_plane0 = 0, out_planes = 0;
};

static bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

static void free_ctx(OocContext &c) {
    if (c.stream) cudaStreamSynchronize(c.stream);
    cudaFree(c.d_mask);
    cudaFree(c.d_out);
    cudaFree(c.ws);
    cudaFreeHost(c.h_in);
    cudaFreeHost(c.h_out);
    if (c.stream) cudaStreamDestroy(c.stream);
    c = OocContext{};
}

}  // namespace maxi

using namespace maxi;

extern "C" int64_t maxi_diffusion_workspace_size(int64_t nz, int64_t ny, int64_t nx, int32_t field_type);

namespace maxi {

// Reads planes [z0, z0 + nzp) of the uint8 mask into `dst` (host memory).
using PlaneReader = std::function<int(int64_t z0, int64_t nzp, uint8_t *dst)>;
// Receives planes [z0, z0 + nzp) of the uint16 output from `src` (host memory).
using PlaneWriter = std::function<int(int64_t z0, int64_t nzp, const uint16_t *src)>;

// The slab engine.  `direct_in` / `direct_out`: pinned caller buffers that the
// device copies can use without staging (may be NULL).
static int run_slabs(int64_t nz, int64_t ny, int64_t nx, int64_t slab_z, const float *kernel, int64_t kernel_size,
                     int64_t repititions, int32_t field_type, int32_t flags, int verbose, const PlaneReader &read,
                     const PlaneWriter &write, const uint8_t *direct_in, uint16_t *direct_out) {
    const int64_t plane = ny * nx;
    const int64_t radius = kernel_size / 2;
    const int64_t halo = std::min(nz, repititions * radius);
    const int64_t S = std::min(slab_z, nz);
    const int64_t E = std::min(nz, S + 2 * halo);  // largest extended slab
    const int64_t n_slabs = ceil_div(nz, S);
    if (verbose >= 1)
        printf("Out-of-core diffusion: shape (%lld, %lld, %lld), %lld slabs of %lld planes, halo %lld planes\n",
               (long long) nz, (long long) ny, (long long) nx, (long long) n_slabs, (long long) S, (long long) halo);

    // Two contexts when they fit in device memory, else one.
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const int64_t ws_bytes = maxi_diffusion_workspace_size(E, ny, nx, field_type);
    if (ws_bytes < 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "unknown field_type %d", field_type);
    const int64_t per_ctx = E * plane * 3 + ws_bytes;
    const int n_ctx = (n_slabs > 1 && (int64_t) free_b > 2 * per_ctx + (int64_t(1) << 30)) ? 2 : 1;

    OocContext ctx[2];
    auto fail = [&](int code) {
        for (auto &c : ctx) free_ctx(c);
        return code;
    };
    for (int c = 0; c < n_ctx; c++) {
        OocContext &x = ctx[c];
        if (cudaStreamCreateWithFlags(&x.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaMalloc(&x.d_mask, E * plane) != cudaSuccess || cudaMalloc(&x.d_out, E * plane * 2) != cudaSuccess ||
            cudaMalloc(&x.ws, ws_bytes) != cudaSuccess ||
            (!direct_in && cudaMallocHost(&x.h_in, E * plane) != cudaSuccess) ||
            (!direct_out && cudaMallocHost(&x.h_out, S * plane * 2) != cudaSuccess)) {
            cudaGetLastError();
            return fail(set_error(MAXI_ERR_OUT_OF_MEMORY,
                                  "could not allocate slab buffers for %lld planes of %lld voxels; use a smaller slab",
                                  (long long) E, (long long) plane));
        }
        x.ws_bytes = ws_bytes;
    }

    // Finishes a context's previous slab: wait for its copy-out, then hand the
    // planes to the writer.
    auto drain = [&](OocContext &x) -> int {
        if (!x.pending) return MAXI_OK;
        cudaError_t e = cudaStreamSynchronize(x.stream);
        if (e != cudaSuccess) return set_cuda_error(e, "out-of-core slab");
        x.pending = false;
        if (!direct_out) return write(x.out_plane0, x.out_planes, x.h_out);
        return MAXI_OK;
    };

    int rc = MAXI_OK;
    for (int64_t s = 0; s < n_slabs; s++) {
        OocContext &x = ctx[s % n_ctx];
        if ((rc = drain(x))) return fail(rc);
        const int64_t z0 = s * S, z1 = std::min(nz, z0 + S);
        const int64_t e0 = std::max<int64_t>(0, z0 - halo), e1 = std::min(nz, z1 + halo);
        const int64_t ez = e1 - e0;
        if (verbose >= 1) printf("\rSlab %lld/%lld", (long long) (s + 1), (long long) n_slabs), fflush(stdout);
        const uint8_t *src = direct_in ? direct_in + e0 * plane : x.h_in;
        if (!direct_in && (rc = read(e0, ez, x.h_in))) return fail(rc);
        cudaError_t e = cudaMemcpyAsync(x.d_mask, src, ez * plane, cudaMemcpyHostToDevice, x.stream);
        if (e != cudaSuccess) return fail(set_cuda_error(e, "slab upload"));
        // A cut side (one that is not the volume's edge) carries a halo of
        // repititions*radius planes, and after repetition k only the planes at
        // least (k+1)*radius away from the cut still hold the whole-volume
        // values: repetition k is computed on those planes alone.
        rc = diffusion_device_shrinking(x.d_mask, MAXI_MASK_U8, ez, ny, nx, kernel, kernel_size, repititions,
                                        x.d_out, nullptr, field_type, flags, x.ws, x.ws_bytes, x.stream,
                                        e0 > 0 ? radius : 0, e1 < nz ? radius : 0);
        if (rc) return fail(rc);
        uint16_t *dst = direct_out ? direct_out + z0 * plane : x.h_out;
        e = cudaMemcpyAsync(dst, x.d_out + (z0 - e0) * plane, (z1 - z0) * plane * 2, cudaMemcpyDeviceToHost, x.stream);
        if (e != cudaSuccess) return fail(set_cuda_error(e, "slab download"));
        x.pending = true;
        x.out_plane0 = z0;
        x.out_planes = z1 - z0;
    }
    for (int c = 0; c < n_ctx; c++)
        if ((rc = drain(ctx[c]))) return fail(rc);
    if (verbose >= 1) printf("\rOut-of-core diffusion is complete!\n");
    fail(0);
    return MAXI_OK;
}

}  // namespace maxi

extern "C" int maxi_diffusion_out_of_core_ex(const uint8_t *voxels, int64_t nz, int64_t ny, int64_t nx,
                                             int64_t slab_z, const float *kernel, int64_t kernel_size,
                                             int64_t repititions, uint16_t *output, int32_t field_type,
                                             int32_t flags, int verbose) {
    clear_error();
    int rc = validate_common(voxels, nz, ny, nx, kernel, kernel_size, repititions);
    if (rc) return rc;
    if (!output) return set_error(MAXI_ERR_INVALID_ARGUMENT, "output is NULL");
    if (slab_z <= 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "slab depth %lld is not positive", (long long) slab_z);
    if ((rc = require_device())) return rc;
    const int64_t plane = ny * nx;
    PlaneReader read = [&](int64_t z0, int64_t nzp, uint8_t *dst) {
        memcpy(dst, voxels + z0 * plane, (size_t) (nzp * plane));
        return MAXI_OK;
    };
    PlaneWriter write = [&](int64_t z0, int64_t nzp, const uint16_t *src) {
        memcpy(output + z0 * plane, src, (size_t) (nzp * plane * 2));
        return MAXI_OK;
    };
    return run_slabs(nz, ny, nx, slab_z, kernel, kernel_size, repititions, field_type, flags, verbose, read, write,
                     is_pinned(voxels) ? voxels : nullptr, is_pinned(output) ? output : nullptr);
}

// On-disk form: replaces NS::diffusion_on_disk (src/lib/cpp/include/diffusion.hh:55,
// GPU body src/lib/cpp/gpu/diffusion.cc:808-945) behind the pybind overload
// src/pybind/diffusion-pybind.cc:67-77.  Reads a raw uint8 volume file and
// writes a raw uint16 file, streaming z-slabs of global_z planes (plus deep
// halos) so neither the host nor the device needs the whole volume.  As in the
// reference, the mask of each repetition is rebuilt from the field
// (`field == 1.0f`, src/lib/cpp/gpu/diffusion.cc:885 / store_mask) and the
// field is FP32; no temporary files are written.
extern "C" int maxi_diffusion_on_disk(const char *input_file, const float *kernel, int64_t kernel_size,
                                      const char *output_file, int64_t total_z, int64_t total_y, int64_t total_x,
                                      int64_t global_z, int64_t global_y, int64_t global_x, int64_t repititions,
                                      int verbose) {
    clear_error();
    if (!input_file || !output_file) return set_error(MAXI_ERR_INVALID_ARGUMENT, "file name is NULL");
    const uint8_t dummy = 0;
    int rc = validate_common(&dummy, total_z, total_y, total_x, kernel, kernel_size, repititions);
    if (rc) return rc;
    if (global_z <= 0 || global_y <= 0 || global_x <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "global_shape must be positive");
    const int64_t plane = total_y * total_x, n = total_z * plane;
    FILE *fin = fopen(input_file, "rb");
    if (!fin) return set_error(MAXI_ERR_IO, "could not open file: %s", input_file);
    if (fseeko(fin, 0, SEEK_END) != 0 || ftello(fin) < n) {
        fclose(fin);
        return set_error(MAXI_ERR_IO, "%s holds fewer than %lld bytes", input_file, (long long) n);
    }
    if ((rc = require_device())) {
        fclose(fin);
        return rc;
    }
    FILE *fout = fopen(output_file, "wb");
    if (!fout) {
        fclose(fin);
        return set_error(MAXI_ERR_IO, "could not open file: %s", output_file);
    }
    PlaneReader read = [&](int64_t z0, int64_t nzp, uint8_t *dst) {
        if (fseeko(fin, (off_t) (z0 * plane), SEEK_SET) != 0 ||
            fread(dst, 1, (size_t) (nzp * plane), fin) != (size_t) (nzp * plane))
            return set_error(MAXI_ERR_IO, "could not read planes %lld..%lld of %s", (long long) z0,
                             (long long) (z0 + nzp), input_file);
        return (int) MAXI_OK;
    };
    PlaneWriter write = [&](int64_t z0, int64_t nzp, const uint16_t *src) {
        if (fseeko(fout, (off_t) (z0 * plane * 2), SEEK_SET) != 0 ||
            fwrite(src, 2, (size_t) (nzp * plane), fout) != (size_t) (nzp * plane))
            return set_error(MAXI_ERR_IO, "could not write planes %lld..%lld of %s", (long long) z0,
                             (long long) (z0 + nzp), output_file);
        return (int) MAXI_OK;
    };
    rc = run_slabs(total_z, total_y, total_x, global_z, kernel, kernel_size, repititions, MAXI_FIELD_F32,
                   MAXI_FLAG_MASK_FROM_FIELD, verbose, read, write, nullptr, nullptr);
    fclose(fin);
    if (fclose(fout) != 0 && rc == MAXI_OK) rc = set_error(MAXI_ERR_IO, "could not close %s", output_file);
    return rc;
}

// Replaces NS::diffusion_out_of_core (src/lib/cpp/include/diffusion.hh:74):
// global_shape gives the slab depth (global_z); the slabs span the full y and
// x extent, so global_y / global_x only have to be positive.
extern "C" int maxi_diffusion_out_of_core(const uint8_t *voxels, int64_t total_z, int64_t total_y, int64_t total_x,
                                          int64_t global_z, int64_t global_y, int64_t global_x, const float *kernel,
                                          int64_t kernel_size, int64_t repititions, uint16_t *output, int verbose) {
    if (global_y <= 0 || global_x <= 0) {
        clear_error();
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "global_shape must be positive");
    }
    return maxi_diffusion_out_of_core_ex(voxels, total_z, total_y, total_x, global_z, kernel, kernel_size,
                                         repititions, output, MAXI_FIELD_F32, 0, verbose);
}
