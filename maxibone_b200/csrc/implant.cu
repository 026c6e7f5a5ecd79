// The implant's solid / shell / front / back masks: the reference's
// compute_front_back_masks (src/lib/cpp/cpu_seq/geometry.cc:112-215, bound by
// src/pybind/geometry-pybind.cc:283-310), which src/processing_steps/0750_bone_region.py:62
// runs to make the `implant_solid` mask that the diffusion step loads and diffuses
// (src/processing_steps/0900_generate_gauss_c.py:49-54,111).
//
// In the implant's frame of reference: uvw = (zyx - cm) @ E per voxel; w0 = the least
// w over the implant's voxels (0 if none is negative); UVW = (uvw - (0, 0, w0)) *
// voxel_size; (Up, Vp, Wp) = (UVW - cp) @ UVWp; r = sqrt(Vp^2 + Wp^2); rmax(z) = the
// largest r * mask over plane z.  Then
//   implant_shell = mask & (r >= 0.7 rmax)        solid_implant = mask | (r < 0.7 rmax && W >= 0)
//   back = W < 0                                   front = (W > 50) & !solid_implant
// with the comparisons against 0.7 rmax in FP64 (0.7 is a double literal there).
//
// Every FP32 operation is rounded on its own, in the reference's order (its x86-64
// build has no fused multiply-add), so the masks are identical.  Three passes over
// the mask: the least w (an order-preserving integer atomicMin), the per-plane rmax
// (atomicMax on the bits of a non-negative float), and the four outputs.
#include "common.cuh"
#include "host_util.h"

namespace maxi {
namespace {

struct Frame {
    float E[9], cm[3], cp[3], P[9], voxel_size;
};

// A float's bits as an int whose signed order is the float's order (no NaNs).
__device__ __forceinline__ int ordered(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7fffffff;
}
__device__ __forceinline__ float from_ordered(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

// (a0 * E[k] + a1 * E[3 + k]) + a2 * E[6 + k], each operation rounded.
__device__ __forceinline__ float dot3(float a0, float a1, float a2, const float *M, int k) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a0, M[k]), __fmul_rn(a1, M[3 + k])), __fmul_rn(a2, M[6 + k]));
}

__device__ __forceinline__ float w_of(const Frame &f, float zf, float yf, float xf) {
    return dot3(__fsub_rn(zf, f.cm[0]), __fsub_rn(yf, f.cm[1]), __fsub_rn(xf, f.cm[2]), f.E, 2);
}

// r and W of voxel (z, y, x).
__device__ __forceinline__ void r_and_W(const Frame &f, float w0, float zf, float yf, float xf, float &r, float &W) {
    const float a0 = __fsub_rn(zf, f.cm[0]), a1 = __fsub_rn(yf, f.cm[1]), a2 = __fsub_rn(xf, f.cm[2]);
    const float U = __fmul_rn(dot3(a0, a1, a2, f.E, 0), f.voxel_size);  // (u - 0) * voxel_size
    const float V = __fmul_rn(dot3(a0, a1, a2, f.E, 1), f.voxel_size);
    W = __fmul_rn(__fsub_rn(dot3(a0, a1, a2, f.E, 2), w0), f.voxel_size);
    const float b0 = __fsub_rn(U, f.cp[0]), b1 = __fsub_rn(V, f.cp[1]), b2 = __fsub_rn(W, f.cp[2]);
    const float Vp = dot3(b0, b1, b2, f.P, 1), Wp = dot3(b0, b1, b2, f.P, 2);
    r = __fsqrt_rn(__fadd_rn(__fmul_rn(Vp, Vp), __fmul_rn(Wp, Wp)));
}

// Blocks walk rows (z, y); threads step along x.
__global__ void implant_least_w(const uint8_t *__restrict__ mask, int64_t nz, int64_t ny, int nx, Frame f,
                                int *__restrict__ w0_key) {
    __shared__ int warp_min[32];
    int best = 0;  // ordered(0.0f): w0 starts at 0
    for (int64_t row = blockIdx.x; row < nz * ny; row += gridDim.x) {
        const int64_t z = row / ny, y = row - z * ny;
        const float zf = (float) z, yf = (float) y;
        const uint8_t *m = mask + row * nx;
        for (int x = threadIdx.x; x < nx; x += blockDim.x)
            if (__ldg(m + x)) {
                const float w = w_of(f, zf, yf, (float) x);
                if (w < 0.0f) best = min(best, ordered(w));  // w0 starts at +0
            }
    }
    for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0) warp_min[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        best = threadIdx.x < (blockDim.x >> 5) ? warp_min[threadIdx.x] : 0;
        for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (threadIdx.x == 0 && best < 0) atomicMin(w0_key, best);
    }
}

// rmax(z) = max over the plane of r * mask (non-negative: its float bits order as ints).
__global__ void implant_plane_rmax(const uint8_t *__restrict__ mask, int64_t nz, int64_t ny, int nx, Frame f,
                                   const int *__restrict__ w0_key, int *__restrict__ rmax_bits) {
    const float w0 = from_ordered(*w0_key);
    for (int64_t row = blockIdx.x; row < nz * ny; row += gridDim.x) {
        const int64_t z = row / ny, y = row - z * ny;
        const float zf = (float) z, yf = (float) y;
        const uint8_t *m = mask + row * nx;
        float best = 0.0f;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            float r, W;
            r_and_W(f, w0, zf, yf, (float) x, r, W);
            best = fmaxf(best, __fmul_rn(r, (float) __ldg(m + x)));
        }
        for (int o = 16; o; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
        if ((threadIdx.x & 31) == 0 && best > 0.0f) atomicMax(rmax_bits + z, __float_as_int(best));
    }
}

__global__ void implant_outputs(const uint8_t *__restrict__ mask, int64_t nz, int64_t ny, int nx, Frame f,
                                const int *__restrict__ w0_key, const int *__restrict__ rmax_bits,
                                uint8_t *__restrict__ front, uint8_t *__restrict__ back,
                                uint8_t *__restrict__ shell, uint8_t *__restrict__ solid) {
    const float w0 = from_ordered(*w0_key);
    for (int64_t row = blockIdx.x; row < nz * ny; row += gridDim.x) {
        const int64_t z = row / ny, y = row - z * ny;
        const float zf = (float) z, yf = (float) y;
        const double lim = __dmul_rn(0.7, (double) __int_as_float(__ldg(rmax_bits + z)));
        const int64_t base = row * nx;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            float r, W;
            r_and_W(f, w0, zf, yf, (float) x, r, W);
            const int m = __ldg(mask + base + x);
            const double rd = (double) r;
            const int so = m | (int) (rd < lim && W >= 0.0f);
            shell[base + x] = (uint8_t) (m & (int) (rd >= lim));
            solid[base + x] = (uint8_t) so;
            back[base + x] = (uint8_t) (W < 0.0f);
            front[base + x] = (uint8_t) ((W > 50.0f) & ((uint8_t) so == 0));
        }
    }
}

}  // namespace
}  // namespace maxi

using namespace maxi;

extern "C" int maxi_implant_masks(const uint8_t *mask, int64_t nz, int64_t ny, int64_t nx, float voxel_size,
                                  const float *E, const float *cm, const float *cp, const float *UVWp,
                                  uint8_t *front_mask, uint8_t *back_mask, uint8_t *implant_shell_mask,
                                  uint8_t *solid_implant, void *stream) {
    clear_error();
    if (!mask || !E || !cm || !cp || !UVWp || !front_mask || !back_mask || !implant_shell_mask || !solid_implant)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (nz <= 0 || ny <= 0 || nx <= 0)
        return set_error(MAXI_ERR_INVALID_ARGUMENT, "shape (%lld, %lld, %lld) has an empty axis", (long long) nz,
                         (long long) ny, (long long) nx);
    if (nz > (int64_t(1) << 24) || ny > (int64_t(1) << 24) || nx > (int64_t(1) << 24))
        return set_error(MAXI_ERR_UNSUPPORTED, "axes longer than 2^24 are not served (coordinates stay exact floats)");
    int rc = require_device();
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    Frame f{};
    for (int i = 0; i < 9; i++) f.E[i] = E[i], f.P[i] = UVWp[i];
    for (int i = 0; i < 3; i++) f.cm[i] = cm[i], f.cp[i] = cp[i];
    f.voxel_size = voxel_size;

    int *scratch = nullptr;  // [0]: ordered least w; [1 ..]: rmax bits per plane
    const size_t bytes = (size_t) (nz + 1) * sizeof(int);
    if (cudaMallocAsync(reinterpret_cast<void **>(&scratch), bytes, st) != cudaSuccess) {
        cudaGetLastError();
        return set_error(MAXI_ERR_OUT_OF_MEMORY, "could not allocate %zu bytes of scratch", bytes);
    }
    cudaError_t e = cudaMemsetAsync(scratch, 0, bytes, st);  // ordered(0.0f) == 0, rmax 0.0f
    if (e == cudaSuccess) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int threads = nx >= 256 ? 256 : 128;
        const unsigned grid = (unsigned) std::min<int64_t>(nz * ny, (int64_t) sms * 16);
        implant_least_w<<<grid, threads, 0, st>>>(mask, nz, ny, (int) nx, f, scratch);
        implant_plane_rmax<<<grid, threads, 0, st>>>(mask, nz, ny, (int) nx, f, scratch, scratch + 1);
        implant_outputs<<<grid, threads, 0, st>>>(mask, nz, ny, (int) nx, f, scratch, scratch + 1, front_mask,
                                                  back_mask, implant_shell_mask, solid_implant);
        e = cudaGetLastError();
    }
    cudaFreeAsync(scratch, st);
    cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "implant masks");
}
