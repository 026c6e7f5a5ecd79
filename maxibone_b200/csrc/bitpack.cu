// Bit-packing of masks: uint8 voxels <-> uint32 words, most significant bit
// first, over the flat voxel order.  The layout of the reference's
// `bitpacking` module (src/lib/cpp/cpu_seq/bitpacking.cc:9-42, GPU form
// src/lib/cpp/gpu/bitpacking.cc:20-145).
//
// encode: each warp packs 32 words (1024 voxels).  Lane l loads 32 bytes of
// its own word as two 16-byte vectors, so a warp reads 1 KiB contiguously.
#include "common.cuh"
#include "host_util.h"

namespace maxi {

// keep_bit0: reference encode semantics (`mask & 1`); otherwise `mask > 0`,
// the diffusion's set test.
template <bool KEEP_BIT0>
__global__ void bitpack_encode_kernel(const uint8_t *__restrict__ mask, int64_t n, uint32_t *__restrict__ packed) {
    const int64_t n_words = (n + 31) / 32;
    for (int64_t w = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; w < n_words;
         w += (int64_t) gridDim.x * blockDim.x) {
        const int64_t base = w * 32;
        uint32_t word = 0;
        if (base + 32 <= n && (reinterpret_cast<uintptr_t>(mask) & 15) == 0) {
            const uint4 *p = reinterpret_cast<const uint4 *>(mask + base);
            const uint4 a = __ldg(p), b = __ldg(p + 1);
            const uint32_t parts[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int q = 0; q < 8; q++) {
#pragma unroll
                for (int by = 0; by < 4; by++) {
                    const uint32_t byte = (parts[q] >> (8 * by)) & 0xffu;
                    const uint32_t bit = KEEP_BIT0 ? (byte & 1u) : (byte != 0u);
                    word |= bit << (31 - (q * 4 + by));
                }
            }
        } else {
            for (int j = 0; j < 32 && base + j < n; j++) {
                const uint32_t byte = mask[base + j];
                const uint32_t bit = KEEP_BIT0 ? (byte & 1u) : (byte != 0u);
                word |= bit << (31 - j);
            }
        }
        packed[w] = word;
    }
}

__global__ void bitpack_decode_kernel(const uint32_t *__restrict__ packed, int64_t n, uint8_t *__restrict__ mask) {
    for (int64_t i = (int64_t) blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t) gridDim.x * blockDim.x) {
        const uint32_t w = __ldg(packed + (i >> 5));
        mask[i] = (uint8_t) ((w >> (31 - (int) (i & 31))) & 1u);
    }
}

cudaError_t launch_bitpack_encode(const uint8_t *mask, int64_t n, uint32_t *packed, bool keep_bit0, cudaStream_t st) {
    const int64_t words = (n + 31) / 32;
    const int64_t blocks = std::min<int64_t>(ceil_div(words, 256), 148 * 32);
    if (keep_bit0) bitpack_encode_kernel<true><<<blocks, 256, 0, st>>>(mask, n, packed);
    else bitpack_encode_kernel<false><<<blocks, 256, 0, st>>>(mask, n, packed);
    return cudaGetLastError();
}

}  // namespace maxi

using namespace maxi;

extern "C" {

int maxi_bitpack_encode(const uint8_t *mask, int64_t n, uint32_t *packed, void *stream) {
    clear_error();
    if (!mask || !packed) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (n < 0 || n % 32 != 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "n = %lld is not a multiple of 32", (long long) n);
    int rc = require_device();
    if (rc) return rc;
    if (n == 0) return MAXI_OK;
    cudaError_t e = launch_bitpack_encode(mask, n, packed, true, static_cast<cudaStream_t>(stream));
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "bitpack encode");
}

int maxi_bitpack_decode(const uint32_t *packed, int64_t n, uint8_t *mask, void *stream) {
    clear_error();
    if (!mask || !packed) return set_error(MAXI_ERR_INVALID_ARGUMENT, "NULL pointer");
    if (n < 0 || n % 32 != 0) return set_error(MAXI_ERR_INVALID_ARGUMENT, "n = %lld is not a multiple of 32", (long long) n);
    int rc = require_device();
    if (rc) return rc;
    if (n == 0) return MAXI_OK;
    const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), 148 * 32);
    bitpack_decode_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(packed, n, mask);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MAXI_OK : set_cuda_error(e, "bitpack decode");
}

}  // extern "C"
