// host_util.h — device and pinned host buffers and small host helpers shared by the engine
// (engine.cu) and the request server (server.cu).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace granite_b200 {

inline int grid_for(int64_t n, int threads) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148 * 64) b = 148 * 64;
    return (int)b;
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t count = 0;
    ~DevBuf() { reset(); }
    void reset() {
        if (p) cudaFree(p);
        p = nullptr;
        count = 0;
    }
    cudaError_t alloc(size_t n) {
        if (n <= count && p) return cudaSuccess;
        reset();
        if (n == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, n * sizeof(T));
        if (e == cudaSuccess) count = n;
        else p = nullptr;
        return e;
    }
};

struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;
    ~PinnedBuf() {
        if (p) cudaFreeHost(p);
        if (done) cudaEventDestroy(done);
    }
};

// Host copy split over up to 8 threads: the staging copies into / out of pinned memory run
// at a few GB/s on one core, which would otherwise set the pace of a run fed from the host.
inline void parallel_memcpy(void *dst, const void *src, size_t bytes) {
    constexpr size_t kMinChunk = size_t(8) << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t t = std::min<size_t>({8, hw, std::max<size_t>(1, bytes / kMinChunk)});
    if (t <= 1) {
        std::memcpy(dst, src, bytes);
        return;
    }
    const size_t chunk = ((bytes + t - 1) / t + 63) & ~size_t(63);
    std::vector<std::thread> pool;
    for (size_t k = 1; k < t; ++k) {
        const size_t off = k * chunk;
        if (off >= bytes) break;
        pool.emplace_back([=] {
            std::memcpy(static_cast<char *>(dst) + off, static_cast<const char *>(src) + off,
                        std::min(chunk, bytes - off));
        });
    }
    std::memcpy(dst, src, std::min(chunk, bytes));
    for (auto &th : pool) th.join();
}

}  // namespace granite_b200
