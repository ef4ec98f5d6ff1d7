// memory.cu — the library's memory caches: page-locked host memory for results and loader data
// (gr_host_*), and the stream-ordered device pool behind every engine, server and field buffer
// (dev_alloc / dev_free, gr_device_cache_*).
//
// The DMA engines move page-locked host memory at the link rate (about 55 GB/s each way on a
// B200 host), while any pageable buffer goes through a host copy into staging first (about
// 20 GB/s with the copy pool), and a freshly allocated pageable buffer also pays its page
// faults on first touch.  Page-locking is itself slow (cudaHostAlloc runs at a few GB/s), so
// freed blocks are kept and handed out again: a loop of runs with results of the same size
// pays it once.  The engine recognises page-locked buffers by their address
// (cudaPointerGetAttributes), whoever allocated them, and then copies without staging.
#include <cuda_runtime.h>
#include <unistd.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/granite_b200.h"

namespace granite_b200 {
void set_last_error(const char *msg);
}

// ------------------------------------------------------------------ device pool
//
// cudaMalloc / cudaFree map and unmap memory on every call; a run that allocates its history
// and ring and frees them at the end pays that each time (tens to hundreds of ms for the GB of
// one run, more when the driver is busy).  Every device buffer of the library instead comes
// from one CUDA memory pool per device whose release threshold is unlimited, so freed memory
// stays mapped and is handed out again.  An allocation that fails trims the pool (returns its
// idle memory to the driver) and retries once.
namespace granite_b200 {
namespace {

constexpr int kMaxDevices = 64;

struct DevicePool {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;   // allocations and frees are ordered on this stream
};

std::mutex g_dev_mu;
DevicePool g_dev[kMaxDevices];

cudaError_t device_pool(int dev, DevicePool *&out) {
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(g_dev_mu);
    DevicePool &d = g_dev[dev];
    if (!d.pool) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool = nullptr;
        cudaError_t err = cudaMemPoolCreate(&pool, &props);
        if (err != cudaSuccess) return err;
        uint64_t keep = UINT64_MAX;
        err = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&d.stream, cudaStreamNonBlocking);
        if (err != cudaSuccess) {
            cudaMemPoolDestroy(pool);
            return err;
        }
        d.pool = pool;
    }
    out = &d;
    return cudaSuccess;
}

}  // namespace

// Device memory of `bytes` on the current device, usable on every stream when this returns.
cudaError_t dev_alloc(void **p, size_t bytes) {
    *p = nullptr;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    DevicePool *d = nullptr;
    err = device_pool(dev, d);
    if (err != cudaSuccess) return err;
    err = cudaMallocFromPoolAsync(p, bytes, d->pool, d->stream);
    if (err == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        cudaStreamSynchronize(d->stream);
        cudaMemPoolTrimTo(d->pool, 0);
        err = cudaMallocFromPoolAsync(p, bytes, d->pool, d->stream);
    }
    if (err != cudaSuccess) {
        *p = nullptr;
        return err;
    }
    return cudaStreamSynchronize(d->stream);
}

// Returns `p` (from dev_alloc) to its device's pool.  Like cudaFree, waits for the device's
// queued work first, so no kernel still in flight can see the memory handed out again.
void dev_free(void *p) {
    if (!p) return;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess || a.type != cudaMemoryTypeDevice) {
        cudaGetLastError();
        return;   // the runtime is unloading, or not ours: nothing safe to do
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (a.device != cur) cudaSetDevice(a.device);
    DevicePool *d = nullptr;
    if (device_pool(a.device, d) == cudaSuccess) {
        cudaDeviceSynchronize();
        cudaFreeAsync(p, d->stream);
        cudaStreamSynchronize(d->stream);
    }
    if (a.device != cur) cudaSetDevice(cur);
}

// Bytes the current device's pool holds mapped but unused (free to the library, not counted
// as free by cudaMemGetInfo).
size_t dev_pool_idle_bytes() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::lock_guard<std::mutex> g(g_dev_mu);
    if (!g_dev[dev].pool) return 0;
    uint64_t reserved = 0, used = 0;
    cudaMemPoolGetAttribute(g_dev[dev].pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(g_dev[dev].pool, cudaMemPoolAttrUsedMemCurrent, &used);
    return reserved > used ? (size_t)(reserved - used) : 0;
}

}  // namespace granite_b200

namespace {

constexpr size_t kGranule = size_t(2) << 20;   // sizes round up to 2 MiB

constexpr size_t kSlot = 4096;   // requests up to this size share slabs of one 2 MiB block

struct HostCache {
    std::mutex mu;
    std::multimap<size_t, void *> free_blocks;   // cached blocks by size
    std::unordered_map<void *, size_t> live;      // blocks handed out, with their sizes
    std::vector<void *> free_slots;               // small requests: 4 KiB slots of slab blocks
    std::unordered_map<void *, char> live_slots;
    size_t cached = 0, live_bytes = 0, limit = 0;
    int64_t allocations = 0, reuses = 0;
    HostCache() {
        // default cache limit: a quarter of the physical memory
        const long pages = sysconf(_SC_PHYS_PAGES), page = sysconf(_SC_PAGESIZE);
        limit = (pages > 0 && page > 0) ? (size_t)pages * (size_t)page / 4 : (size_t(16) << 30);
    }
};

// Never destroyed: numpy arrays that own blocks may be released after static destruction.
HostCache &cache() {
    static HostCache *c = new HostCache;
    return *c;
}

int host_fail(int code, const std::string &msg) {
    granite_b200::set_last_error(msg.c_str());
    return code;
}

// Frees cached blocks (largest first) until at most `keep` bytes stay cached.  Called without
// the lock held: cudaFreeHost may wait for the device.
void release_cached(size_t keep) {
    std::vector<void *> drop;
    {
        HostCache &c = cache();
        std::lock_guard<std::mutex> g(c.mu);
        while (c.cached > keep && !c.free_blocks.empty()) {
            auto it = std::prev(c.free_blocks.end());
            c.cached -= it->first;
            drop.push_back(it->second);
            c.free_blocks.erase(it);
        }
    }
    for (void *p : drop) cudaFreeHost(p);
}

}  // namespace

extern "C" {

int gr_host_alloc(int64_t bytes, void **out) {
    if (!out) return host_fail(GR_ERR_USER, "ERROR < USER INPUT | null argument >");
    *out = nullptr;
    if (bytes < 0) return host_fail(GR_ERR_USER, "ERROR < USER INPUT | negative size >");
    if (bytes == 0) return GR_OK;
    HostCache &c = cache();
    if ((size_t)bytes <= kSlot) {
        // small words (counters, flags) share slabs: one page-locked block serves 512 of them
        std::lock_guard<std::mutex> g(c.mu);
        if (c.free_slots.empty()) {
            void *slab = nullptr;
            const cudaError_t err = cudaHostAlloc(&slab, kGranule, cudaHostAllocPortable);
            if (err != cudaSuccess) {
                cudaGetLastError();
                return host_fail(GR_ERR_RUNTIME, std::string("ERROR < RUNTIME | CUDA error | ") +
                                                     cudaGetErrorString(err) + " : page-locked slab >");
            }
            ++c.allocations;
            for (size_t k = kGranule / kSlot; k-- > 0;) c.free_slots.push_back(static_cast<char *>(slab) + k * kSlot);
        }
        *out = c.free_slots.back();
        c.free_slots.pop_back();
        c.live_slots.emplace(*out, 0);
        c.live_bytes += kSlot;
        return GR_OK;
    }
    const size_t need = ((size_t)bytes + kGranule - 1) / kGranule * kGranule;
    {
        // smallest cached block that fits, unless it is more than a quarter larger
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.free_blocks.lower_bound(need);
        if (it != c.free_blocks.end() && it->first <= need + need / 4) {
            *out = it->second;
            c.cached -= it->first;
            c.live_bytes += it->first;
            c.live.emplace(it->second, it->first);
            c.free_blocks.erase(it);
            ++c.reuses;
            return GR_OK;
        }
    }
    void *p = nullptr;
    cudaError_t err = cudaHostAlloc(&p, need, cudaHostAllocPortable);
    if (err != cudaSuccess) {
        cudaGetLastError();
        release_cached(0);   // page-locked memory is scarce: give back the cache and retry once
        err = cudaHostAlloc(&p, need, cudaHostAllocPortable);
        if (err != cudaSuccess) {
            cudaGetLastError();
            return host_fail(GR_ERR_RUNTIME, std::string("ERROR < RUNTIME | CUDA error | ") +
                                                 cudaGetErrorString(err) + " : page-locked allocation of " +
                                                 std::to_string(need) + " bytes >");
        }
    }
    std::lock_guard<std::mutex> g(c.mu);
    c.live.emplace(p, need);
    c.live_bytes += need;
    ++c.allocations;
    *out = p;
    return GR_OK;
}

int gr_host_free(void *p) {
    if (!p) return GR_OK;
    HostCache &c = cache();
    size_t size = 0;
    bool keep = false;
    {
        std::lock_guard<std::mutex> g(c.mu);
        auto sl = c.live_slots.find(p);
        if (sl != c.live_slots.end()) {
            c.live_slots.erase(sl);
            c.free_slots.push_back(p);
            c.live_bytes -= kSlot;
            return GR_OK;
        }
        auto it = c.live.find(p);
        if (it == c.live.end())
            return host_fail(GR_ERR_USER, "ERROR < USER INPUT | gr_host_free: pointer not from gr_host_alloc >");
        size = it->second;
        c.live.erase(it);
        c.live_bytes -= size;
        if (c.cached + size <= c.limit) {
            c.free_blocks.emplace(size, p);
            c.cached += size;
            keep = true;
        }
    }
    if (!keep) cudaFreeHost(p);   // errors ignored: the runtime may already be unloading
    return GR_OK;
}

int gr_host_cache_limit(int64_t bytes) {
    if (bytes < 0) return host_fail(GR_ERR_USER, "ERROR < USER INPUT | negative size >");
    {
        HostCache &c = cache();
        std::lock_guard<std::mutex> g(c.mu);
        c.limit = (size_t)bytes;
    }
    release_cached((size_t)bytes);
    return GR_OK;
}

int gr_host_cache_trim(void) {
    release_cached(0);
    return GR_OK;
}

int gr_host_cache_stats_get(gr_host_cache_stats *out) {
    if (!out) return host_fail(GR_ERR_USER, "ERROR < USER INPUT | null argument >");
    HostCache &c = cache();
    std::lock_guard<std::mutex> g(c.mu);
    out->live_bytes = (int64_t)c.live_bytes;
    out->cached_bytes = (int64_t)c.cached;
    out->limit_bytes = (int64_t)c.limit;
    out->allocations = c.allocations;
    out->reuses = c.reuses;
    return GR_OK;
}

int gr_device_cache_stats_get(int32_t device, int64_t *reserved_bytes, int64_t *used_bytes) {
    if (!reserved_bytes || !used_bytes) return host_fail(GR_ERR_USER, "ERROR < USER INPUT | null argument >");
    *reserved_bytes = *used_bytes = 0;
    if (device < 0 || device >= granite_b200::kMaxDevices)
        return host_fail(GR_ERR_USER, "ERROR < USER INPUT | invalid device >");
    std::lock_guard<std::mutex> g(granite_b200::g_dev_mu);
    cudaMemPool_t pool = granite_b200::g_dev[device].pool;
    if (!pool) return GR_OK;
    uint64_t r = 0, u = 0;
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &r);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &u);
    *reserved_bytes = (int64_t)r;
    *used_bytes = (int64_t)u;
    return GR_OK;
}

int gr_device_cache_trim(void) {
    std::lock_guard<std::mutex> g(granite_b200::g_dev_mu);
    for (auto &d : granite_b200::g_dev) {
        if (!d.pool) continue;
        cudaStreamSynchronize(d.stream);
        cudaMemPoolTrimTo(d.pool, 0);
    }
    return GR_OK;
}

int gr_host_is_pinned(const void *p) {
    if (!p) return 0;
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return a.type == cudaMemoryTypeHost ? 1 : 0;
}

}  // extern "C"
