// batch.cu — several engines' runs as one CUDA graph (gr_batch_*, include/granite_b200.h).
//
// No counterpart in the reference, which runs one TrajectoryIntegrator at a time and launches
// once per step.  Here each engine's whole run over its resident snapshots (seeding, every
// step launch, the compaction / re-sort passes, the final records) is enqueued with fixed
// launch shapes on the engine's own stream.  The streams fork from the batch stream and join
// it again inside one stream capture, so the engines' runs overlap on the device and a replay
// costs one graph launch.
#include <cuda_runtime.h>

#include <cstdio>
#include <string>
#include <vector>

#include "../../include/granite_b200.h"
#include "engine_graph.h"

using namespace granite_b200;

struct gr_batch {
    std::vector<gr_engine *> engines;
    std::vector<uint64_t> gens;          // engine generations the graph was captured for
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> joins;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    gr_batch_stats stats{};

    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~gr_batch() {
        if (stream) cudaStreamSynchronize(stream);
        drop_graph();
        for (auto e : joins) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int batch_fail(int code, const std::string &msg) {
    set_last_error(msg.c_str());
    return code;
}

#define BK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t err_ = (call);                                                                 \
        if (err_ != cudaSuccess) {                                                                 \
            char buf_[256];                                                                        \
            snprintf(buf_, sizeof buf_, "ERROR < RUNTIME | CUDA error | %s : %s, line %d >",       \
                     cudaGetErrorString(err_), __FILE__, __LINE__);                                \
            return batch_fail(GR_ERR_RUNTIME, buf_);                                               \
        }                                                                                          \
    } while (0)

bool stale(const gr_batch *b) {
    if (!b->exec) return true;
    for (size_t i = 0; i < b->engines.size(); ++i)
        if (engine_generation(b->engines[i]) != b->gens[i]) return true;
    return false;
}

// Ends a capture that failed half-way, so the streams are usable again.
void abort_capture(gr_batch *b) {
    cudaGraph_t g = nullptr;
    cudaStreamEndCapture(b->stream, &g);
    if (g) cudaGraphDestroy(g);
    cudaGetLastError();
}

int capture(gr_batch *b) {
    b->drop_graph();
    for (gr_engine *e : b->engines) {
        const int rc = graph_prepare(e);
        if (rc) return rc;
    }
    BK(cudaSetDevice(b->device));
    BK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    cudaError_t err = cudaEventRecord(b->fork, b->stream);
    int rc = GR_OK;
    int64_t launches = 0, aux = 0;
    for (size_t i = 0; i < b->engines.size() && err == cudaSuccess && rc == GR_OK; ++i) {
        gr_engine *e = b->engines[i];
        cudaStream_t s = engine_stream(e);
        err = cudaStreamWaitEvent(s, b->fork, 0);
        if (err != cudaSuccess) break;
        rc = graph_enqueue(e);
        if (rc) break;
        err = cudaEventRecord(b->joins[i], s);
        if (err != cudaSuccess) break;
        err = cudaStreamWaitEvent(b->stream, b->joins[i], 0);
        int64_t a = 0;
        launches += engine_launches(e, &a);
        aux += a;
    }
    if (err != cudaSuccess || rc != GR_OK) {
        std::string msg = rc ? std::string(gr_last_error()) : std::string(cudaGetErrorString(err));
        abort_capture(b);
        return batch_fail(rc ? rc : GR_ERR_RUNTIME, rc ? msg : "ERROR < RUNTIME | CUDA error | " + msg + " >");
    }
    BK(cudaStreamEndCapture(b->stream, &b->graph));
    BK(cudaGraphInstantiate(&b->exec, b->graph, 0));
    size_t nodes = 0;
    BK(cudaGraphGetNodes(b->graph, nullptr, &nodes));
    b->stats.nodes = (int64_t)nodes;
    b->stats.kernel_launches = launches;
    b->stats.aux_launches = aux;
    b->stats.captures++;
    for (size_t i = 0; i < b->engines.size(); ++i) b->gens[i] = engine_generation(b->engines[i]);
    return GR_OK;
}

}  // namespace

extern "C" {

int gr_batch_create(gr_engine *const *engines, int32_t n, gr_batch **out) {
    if (!engines || !out || n <= 0) return batch_fail(GR_ERR_USER, "ERROR < USER INPUT | empty batch >");
    *out = nullptr;
    auto b = new gr_batch();
    for (int32_t i = 0; i < n; ++i) {
        if (!engines[i]) {
            delete b;
            return batch_fail(GR_ERR_USER, "ERROR < USER INPUT | null engine in batch >");
        }
        for (gr_engine *o : b->engines)
            if (o == engines[i]) {
                delete b;
                return batch_fail(GR_ERR_USER, "ERROR < USER INPUT | an engine appears twice in a batch >");
            }
        if (i > 0 && engine_device(engines[i]) != engine_device(engines[0])) {
            delete b;
            return batch_fail(GR_ERR_USER, "ERROR < USER INPUT | the engines of a batch must use one device >");
        }
        b->engines.push_back(engines[i]);
    }
    b->gens.assign(b->engines.size(), 0);
    b->device = engine_device(engines[0]);
    cudaError_t err = cudaSetDevice(b->device);
    if (err == cudaSuccess) err = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaEventCreate(&b->t0);
    if (err == cudaSuccess) err = cudaEventCreate(&b->t1);
    b->joins.assign(b->engines.size(), nullptr);
    for (auto &j : b->joins)
        if (err == cudaSuccess) err = cudaEventCreateWithFlags(&j, cudaEventDisableTiming);
    if (err != cudaSuccess) {
        delete b;
        return batch_fail(GR_ERR_RUNTIME, std::string("ERROR < RUNTIME | CUDA error | ") + cudaGetErrorString(err) + " >");
    }
    *out = b;
    return GR_OK;
}

void gr_batch_destroy(gr_batch *b) { delete b; }

int gr_batch_run(gr_batch *b) {
    if (!b) return batch_fail(GR_ERR_USER, "ERROR < USER INPUT | null batch >");
    BK(cudaSetDevice(b->device));
    if (stale(b)) {
        const int rc = capture(b);
        if (rc) return rc;
    }
    BK(cudaEventRecord(b->t0, b->stream));
    BK(cudaGraphLaunch(b->exec, b->stream));
    BK(cudaEventRecord(b->t1, b->stream));
    BK(cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    BK(cudaEventElapsedTime(&ms, b->t0, b->t1));
    b->stats.graph_ms = ms;
    b->stats.replays++;
    int64_t ps = 0;
    for (gr_engine *e : b->engines) {
        const int rc = graph_collect(e);
        if (rc) return rc;
        ps += engine_particle_steps(e);
    }
    b->stats.particle_steps = ps;
    return GR_OK;
}

int gr_batch_stats_get(const gr_batch *b, gr_batch_stats *out) {
    if (!b || !out) return batch_fail(GR_ERR_USER, "ERROR < USER INPUT | null argument >");
    *out = b->stats;
    return GR_OK;
}

}  // extern "C"
