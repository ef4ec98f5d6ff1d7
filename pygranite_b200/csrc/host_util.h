// host_util.h — device and pinned host buffers and small host helpers shared by the engine
// (engine.cu) and the request server (server.cu).
#pragma once

#include <cuda_runtime.h>

#include "copy_pool.h"
#include "../../include/granite_b200.h"

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace granite_b200 {

// Device memory from the library's per-device pool (memory.cu): freed blocks stay mapped and
// are reused, so repeated runs do not pay cudaMalloc / cudaFree.
cudaError_t dev_alloc(void **p, size_t bytes);
void dev_free(void *p);
size_t dev_pool_idle_bytes();

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
        if (p) dev_free(p);
        p = nullptr;
        count = 0;
    }
    cudaError_t alloc(size_t n) {
        if (n <= count && p) return cudaSuccess;
        reset();
        if (n == 0) return cudaSuccess;
        cudaError_t e = dev_alloc(reinterpret_cast<void **>(&p), n * sizeof(T));
        if (e == cudaSuccess) count = n;
        else p = nullptr;
        return e;
    }
};

// Page-locked staging from the library's host cache (gr_host_alloc): engines created one after
// another reuse the same blocks instead of page-locking and unlocking memory each time.
struct PinnedBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaEvent_t done = nullptr;
    ~PinnedBuf() {
        if (p) gr_host_free(p);
        if (done) cudaEventDestroy(done);
    }
};

}  // namespace granite_b200
