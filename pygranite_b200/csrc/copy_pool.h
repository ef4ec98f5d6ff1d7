// copy_pool.h — large host copies on a persistent pool of worker threads (no CUDA), shared by
// the engine's pinned staging (host_util.h) and the Python module's result accessors.
#pragma once

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

// Host copies into and out of pinned staging, split into 1 MB chunks over a persistent pool of
// worker threads (at most 16, created on first use) and the calling thread.  One core copies a
// few GB/s, which would otherwise set the pace of a run fed from host memory.
class CopyPool {
  public:
    static CopyPool &get() {
        static CopyPool pool;
        return pool;
    }

    void copy(void *dst, const void *src, size_t bytes) {
        constexpr size_t kChunk = size_t(1) << 20;
        const size_t chunks = (bytes + kChunk - 1) / kChunk;
        if (chunks <= 1 || workers_.empty()) {
            std::memcpy(dst, src, bytes);
            return;
        }
        // each job has its own counters: a worker still holding an earlier job finds it exhausted
        auto job = std::make_shared<Job>();
        job->dst = static_cast<char *>(dst);
        job->src = static_cast<const char *>(src);
        job->bytes = bytes;
        job->chunk = kChunk;
        job->chunks = chunks;
        std::unique_lock<std::mutex> lk(mu_);
        busy_cv_.wait(lk, [&] { return !job_; });   // one job at a time
        job_ = job;
        ++generation_;
        lk.unlock();
        work_cv_.notify_all();
        run(*job);
        lk.lock();
        done_cv_.wait(lk, [&] { return job->done.load() == job->chunks; });
        job_.reset();
        lk.unlock();
        busy_cv_.notify_one();
    }

    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(mu_);
            stop_ = true;
        }
        work_cv_.notify_all();
        for (auto &t : workers_) t.join();
    }

  private:
    struct Job {
        char *dst = nullptr;
        const char *src = nullptr;
        size_t bytes = 0, chunk = 0, chunks = 0;
        std::atomic<size_t> next{0}, done{0};
    };

    CopyPool() {
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const unsigned n = std::min(15u, hw > 1 ? hw - 1 : 0u);   // plus the caller: at most 16
        for (unsigned k = 0; k < n; ++k) workers_.emplace_back([this] { loop(); });
    }

    void run(Job &job) {
        for (;;) {
            const size_t c = job.next.fetch_add(1);
            if (c >= job.chunks) return;
            const size_t off = c * job.chunk;
            std::memcpy(job.dst + off, job.src + off, std::min(job.chunk, job.bytes - off));
            if (job.done.fetch_add(1) + 1 == job.chunks) {
                std::lock_guard<std::mutex> g(mu_);
                done_cv_.notify_all();
            }
        }
    }

    void loop() {
        uint64_t seen = 0;
        for (;;) {
            std::shared_ptr<Job> job;
            {
                std::unique_lock<std::mutex> lk(mu_);
                work_cv_.wait(lk, [&] { return stop_ || (job_ && generation_ != seen); });
                if (stop_) return;
                seen = generation_;
                job = job_;
            }
            run(*job);
        }
    }

    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable work_cv_, done_cv_, busy_cv_;
    std::shared_ptr<Job> job_;
    bool stop_ = false;
    uint64_t generation_ = 0;
};

inline void parallel_memcpy(void *dst, const void *src, size_t bytes) { CopyPool::get().copy(dst, src, bytes); }

}  // namespace granite_b200
