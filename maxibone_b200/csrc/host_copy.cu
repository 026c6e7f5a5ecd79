// Staged host <-> device copies for pageable caller buffers (host_copy.h).
#include "host_copy.h"

#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

namespace maxi {

namespace {

constexpr size_t kChunk = size_t(32) << 20;  // bytes per staging buffer

// memcpy split over up to `threads` host threads (contiguous 64 KB-aligned slices).
void parallel_memcpy(void *dst, const void *src, size_t n, int threads) {
    const size_t min_slice = size_t(4) << 20;
    int t = (int) std::min<size_t>((size_t) threads, std::max<size_t>(1, n / min_slice));
    if (t <= 1) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t slice = ((n + t - 1) / t + 65535) & ~size_t(65535);
    std::vector<std::thread> pool;
    pool.reserve(t);
    size_t done = 0;  // bytes handed to threads; the rest is copied here
    try {
        for (int i = 0; i < t; i++) {
            const size_t off = (size_t) i * slice;
            if (off >= n) break;
            const size_t len = std::min(slice, n - off);
            pool.emplace_back([=]() {
                std::memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off, len);
            });
            done = off + len;
        }
    } catch (...) {
        // no more threads: this thread copies what is left
    }
    if (done < n) std::memcpy(static_cast<char *>(dst) + done, static_cast<const char *>(src) + done, n - done);
    for (auto &th : pool) th.join();
}

int copy_threads() {
    const unsigned hc = std::thread::hardware_concurrency();
    return (int) std::max(1u, std::min(16u, hc ? hc : 1u));
}

// Two pinned staging buffers and their "DMA done" events, released on scope exit.
struct Staging {
    void *buf[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    cudaError_t init(size_t bytes) {
        for (int i = 0; i < 2; i++) {
            cudaError_t e = cudaHostAlloc(&buf[i], bytes, cudaHostAllocDefault);
            if (e != cudaSuccess) return e;
            if ((e = cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }
    ~Staging() {
        for (int i = 0; i < 2; i++) {
            if (ev[i]) {
                cudaEventSynchronize(ev[i]);
                cudaEventDestroy(ev[i]);
            }
            if (buf[i]) cudaFreeHost(buf[i]);
        }
    }
};

}  // namespace

bool host_pageable(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeUnregistered;
}

cudaError_t copy_to_device_staged(void *d_dst, const void *h_src, size_t n, cudaStream_t st) {
    Staging s;
    cudaError_t e = s.init(std::min(n, kChunk));
    if (e != cudaSuccess) return e;
    const int threads = copy_threads();
    size_t k = 0;
    for (size_t off = 0; off < n; off += kChunk, k++) {
        const int b = (int) (k & 1);
        const size_t len = std::min(kChunk, n - off);
        // the buffer's previous chunk (k - 2) has crossed to the device
        if (k >= 2 && (e = cudaEventSynchronize(s.ev[b])) != cudaSuccess) return e;
        parallel_memcpy(s.buf[b], static_cast<const char *>(h_src) + off, len, threads);
        if ((e = cudaMemcpyAsync(static_cast<char *>(d_dst) + off, s.buf[b], len, cudaMemcpyHostToDevice, st)) !=
                cudaSuccess ||
            (e = cudaEventRecord(s.ev[b], st)) != cudaSuccess)
            return e;
    }
    return cudaStreamSynchronize(st);
}

cudaError_t copy_to_host_staged(void *h_dst, const void *d_src, size_t n, cudaStream_t st) {
    Staging s;
    cudaError_t e = s.init(std::min(n, kChunk));
    if (e != cudaSuccess) return e;
    const int threads = copy_threads();
    const size_t chunks = (n + kChunk - 1) / kChunk;
    // chunk k -> buffer k & 1; the host empties chunk k - 1 while chunk k crosses
    for (size_t k = 0; k <= chunks; k++) {
        if (k < chunks) {
            const int b = (int) (k & 1);
            const size_t off = k * kChunk, len = std::min(kChunk, n - off);
            if ((e = cudaMemcpyAsync(s.buf[b], static_cast<const char *>(d_src) + off, len, cudaMemcpyDeviceToHost,
                                     st)) != cudaSuccess ||
                (e = cudaEventRecord(s.ev[b], st)) != cudaSuccess)
                return e;
        }
        if (k >= 1) {
            const int b = (int) ((k - 1) & 1);
            const size_t off = (k - 1) * kChunk, len = std::min(kChunk, n - off);
            if ((e = cudaEventSynchronize(s.ev[b])) != cudaSuccess) return e;
            parallel_memcpy(static_cast<char *>(h_dst) + off, s.buf[b], len, threads);
        }
    }
    return cudaSuccess;
}

}  // namespace maxi
