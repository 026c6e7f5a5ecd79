// Host interface of the multi-volume tensor-core passes (tc_batch.cu).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "tc_pass.h"

namespace maxi {
namespace tc {

// Device-table entry of one volume: tensor maps of the pass inputs
// ([pass z/y/x][buffer]), of the y pass's stores, of the z pass's input in
// [y][z][x] row order and of the fused y + x kernel's stores in that order
// ([buffer]), the two ping-pong field buffers, the bit-packed mask, the final
// outputs and the tile counts.
struct alignas(64) TcVol {
    CUtensorMap map[3][2];
    CUtensorMap ystore[2];
    CUtensorMap zrows[2];   // z-pass input read as [y][z][x] rows ([buffer])
    CUtensorMap yxrows[2];  // fused y + x stores to [y][z][x] rows ([buffer]), box 32 x 1 x 32
    void *buf[2];
    const uint32_t *mask;
    uint16_t *out_u16;
    float *field_out;
    int64_t nz, ny, nx;
    int n_at_z, n_at_y, n_xc_z, n_xc_y, n_xt;
    int64_t cols_z, cols_y, tiles_x, tiles_yx;
    uint64_t magic_xt, magic_at_y;  // fused kernel's tile decode: divisions by n_xt and n_at_y
};

// K extents of the strided (z/y) and contiguous (x) tensor-core passes.
struct TcGeometry {
    int radius, kp_strided, kpa_strided, ra, kp_contig, kpa_contig;
};

TcGeometry tc_geometry(int radius);
PFN_cuTensorMapEncodeTiled_v12000 tc_encode_fn();
// Splits float taps (times `scale`) into high and low 16-bit halves.
void tc_split_taps(const float *kernel, int radius, bool is_bf16, float scale, uint16_t *hi, uint16_t *lo);

int tc_fill_volume(TcVol &vol, void *buf0, void *buf1, const uint32_t *packed_mask, uint16_t *out_u16,
                   float *field_out, int64_t nz, int64_t ny, int64_t nx, bool is_bf16, const TcGeometry &g);

// One pass (0 z, 1 y, 2 x, 3 fused y + x) over all volumes of a device table;
// d_prefix holds n_vol + 1 prefix sums of the volumes' columns (z: cols_z, y:
// cols_y) or tiles (x: tiles_x, fused: tiles_yx).  The fused pass needs the
// single coefficient set (hi_only) and radius <= kTcMaxRadius.
// rows_yz: the z pass reads its input as [y][z][x] rows, the x pass (not
// final) writes its output in that order.  hi_only: one matched 16-bit
// coefficient set (the default of the single-volume passes) instead of the
// high and low halves.
cudaError_t tc_batch_pass(const TcVol *d_vols, const int64_t *d_prefix, int64_t total, int n_vol, int pass, int in_buf,
                          bool final_pass, const float *kernel, const TcGeometry &g, bool is_bf16, bool error_feedback,
                          bool rows_yz, cudaStream_t st, bool hi_only);

int tc_batch_read_and_clear_error();

}  // namespace tc
}  // namespace maxi
