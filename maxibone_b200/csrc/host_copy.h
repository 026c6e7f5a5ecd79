// Copies between a caller's pageable host buffer and device memory through two
// pinned staging buffers, several host threads moving each chunk between the
// caller's pages and the pinned buffer while the previous chunk crosses PCIe.
// maxibone's callers hand the drop-in call np.empty arrays (pageable, their
// pages not yet touched): a plain cudaMemcpy from such memory stages through
// the driver's buffers with one host thread, and the first write of every page
// faults on that thread.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace maxi {

// True when `p` is ordinary pageable host memory (not pinned or registered
// with CUDA, not device or managed memory).
bool host_pageable(const void *p);

// h_src (pageable, n bytes) -> d_dst; returns once the data is on the device.
cudaError_t copy_to_device_staged(void *d_dst, const void *h_src, size_t n, cudaStream_t st);

// d_src -> h_dst (pageable, n bytes); returns once the data is in h_dst.  The
// stream's earlier work (the kernels that wrote d_src) completes first.
cudaError_t copy_to_host_staged(void *h_dst, const void *d_src, size_t n, cudaStream_t st);

}  // namespace maxi
