// server.cu — the trajectory request server (gr_server_*, include/granite_b200.h).
//
// No counterpart in the reference, which integrates one seed set per TrajectoryIntegrator.
// Requests (a seed set, a start time, a step count, Euler or RK4) arrive at any time from
// any thread.  One worker thread sweeps the field window by window: a 4-slot device ring
// holds the snapshots of the current window and the next ones, refilled from pinned host
// memory on a copy stream while the current window integrates.  All requests share the
// field's global step clock (start times are rounded down to the step grid), so the particles of
// every request active in a window advance in the same launch (continuous batching):
//
//   per window, on the compute stream:
//     admit   requests whose start step falls in the window, while their state fits the
//             HBM budget: seeds -> the tail of the integrator's particle pool;
//     pack    the window-pair buffer from the two ring slots (planar, unpadded on the host
//             and in the ring: 25% less upload than padded 3D nodes);
//     advance one persistent grid-stride launch per pool over the window's steps (a
//             particle runs steps [start, end) of the clock);
//     retire  compaction + Morton re-sort of each pool; particles that aborted or reached
//             their end step leave the pool, their final state written to their request's
//             slots of the result arena;
//     return  requests whose end step is in the window are complete: their result slices
//             go to pinned host memory, and the worker hands them out when the copy is done.
//
// With no particle in flight the sweep jumps to the earliest start window waiting.  A
// request whose start window the sweep has passed waits for the next sweep.  Per-particle
// arithmetic depends only on the particle and the clock, so a request's result is the same
// alone and in any mix of other requests.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/granite_b200.h"
#include "advance.h"
#include "compact.cuh"
#include "engine_graph.h"
#include "host_util.h"
#include "schedule.h"

using namespace granite_b200;

namespace {

constexpr int kRing = 4;         // ring slots
constexpr int kLag = 2;          // windows the host may enqueue ahead of the device

// First-fit allocator of index ranges (result arena, pinned staging).
class RangeAlloc {
  public:
    void reset(int64_t size) {
        free_.clear();
        if (size > 0) free_[0] = size;
    }
    int64_t take(int64_t n) {
        for (auto it = free_.begin(); it != free_.end(); ++it)
            if (it->second >= n) {
                const int64_t off = it->first, len = it->second;
                free_.erase(it);
                if (len > n) free_[off + n] = len - n;
                return off;
            }
        return -1;
    }
    void give(int64_t off, int64_t n) {
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }

  private:
    std::map<int64_t, int64_t> free_;
};

struct Pool {
    struct Arrays {
        DevBuf<float> px, py, pz;
        DevBuf<int32_t> status, id, life, birth;
    };
    Arrays st[2];
    int cur = 0;
    int64_t cap = 0;                   // particle slots
    int64_t in_flight = 0;             // particles of active requests (upper bound of the live count)
    DevBuf<int32_t> counts;            // [0] live, [1] live after a pass, [2] retired
    DevBuf<int32_t> key, perm;
    AdvanceFn fn = nullptr;
    int threads = 256;
    int64_t grid = 1;
};

struct Req {
    int64_t id = 0;
    int32_t integrator = 1;
    int64_t n = 0;
    int64_t start_step = 0, end_step = 0, start_window = 0;
    int64_t slot = -1;                 // result arena offset
    int64_t stage = -1;                // pinned staging offset (floats)
    std::vector<float> seeds;
    std::vector<float> pos;
    std::vector<int32_t> status;
    double t_submit = 0, t_admit = 0, t_done = 0;
    int32_t state = GR_REQ_PENDING;
    bool cancelled = false;
    bool ended = false;                // its particles have all retired; results wait for staging
    cudaEvent_t done_ev = nullptr;
};

}  // namespace

struct gr_server {
    gr_settings s{};
    int dim = 3;
    int64_t nx = 0, ny = 0, nz = 1, nodes = 0;
    float scale[3]{}, off[3]{}, dom[3]{}, inv_scale[3]{};
    int64_t n_snap = 0, W = 0;
    Schedule sched;
    DevBuf<StepEntry> d_sched;
    int64_t elem = 4;                  // bytes per stored value
    std::vector<void *> host_snap;     // pinned packed snapshots
    int64_t snap_bytes = 0, slot_stride = 0;
    DevBuf<char> ring, pair;
    DevBuf<float> raw;
    int64_t ring_holds[kRing];
    bool slot_used[kRing]{};
    cudaEvent_t slot_ready[kRing]{}, slot_free[kRing]{};
    std::vector<cudaEvent_t> win_done;   // kLag + 1 events: windows in flight
    int64_t win_count = 0;

    Pool pools[2];                     // [0] Euler, [1] RK4
    DevBuf<float> res_px, res_py, res_pz;
    DevBuf<int32_t> res_status;
    int64_t arena_cap = 0;
    RangeAlloc arena;
    float *pin_res = nullptr;          // pinned result staging
    int64_t pin_res_cap = 0;           // floats
    RangeAlloc pin_alloc;
    struct Stage {                     // admission staging, two used in turn
        float *h = nullptr;            // pinned: seeds, then id / end step / start step
        int64_t cap = 0;               // particles
        cudaEvent_t ev = nullptr;      // its last upload
        DevBuf<float> seeds;
        DevBuf<int32_t> meta;
    };
    Stage stage[2];
    int stage_next = 0;
    DevBuf<int32_t> bintab, hist, chunk;
    int bx = 4, by = 4, bz = 2, nbx = 0, nby = 0, nbz = 0, nbins = 0;
    DevBuf<unsigned long long> counters;   // [0] particle-steps
    cudaStream_t cs = nullptr, xs = nullptr;

    std::thread worker;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    bool stop = false, started = false;
    std::deque<int64_t> pending;       // request ids in arrival order
    std::map<int64_t, std::unique_ptr<Req>> reqs;
    std::vector<int64_t> active, returning;
    int64_t next_id = 1;
    int64_t sweep = 0, w = 0;
    std::string failure;
    gr_server_stats st{};
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();

    double now() const {
        return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    ~gr_server();
};

namespace {

int sfail(int code, const std::string &msg) {
    set_last_error(msg.c_str());
    return code;
}

#define SUSER(msg) sfail(GR_ERR_USER, std::string("ERROR < USER INPUT | ") + (msg) + " >")

#define SK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t err_ = (call);                                                                 \
        if (err_ != cudaSuccess) {                                                                 \
            char buf_[256];                                                                        \
            snprintf(buf_, sizeof buf_, "ERROR < RUNTIME | CUDA error | %s : %s, line %d >",       \
                     cudaGetErrorString(err_), __FILE__, __LINE__);                                \
            return sfail(GR_ERR_RUNTIME, buf_);                                                    \
        }                                                                                          \
    } while (0)

// Admitted particles -> the tail of a pool (live prefix), one thread per particle.
__global__ void append_kernel(const float *__restrict__ seeds, const int32_t *__restrict__ meta, int64_t m,
                              int dim, const int32_t *n_act, float *px, float *py, float *pz, int32_t *status,
                              int32_t *id, int32_t *life, int32_t *birth) {
    const int64_t base = *n_act;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = base + i;
        px[d] = seeds[i * dim];
        py[d] = seeds[i * dim + 1];
        if (dim == 3) pz[d] = seeds[i * dim + 2];
        status[d] = 0;
        id[d] = meta[i];
        life[d] = meta[m + i];
        birth[d] = meta[2 * m + i];
    }
}

__global__ void grow_kernel(int32_t *counts, int32_t m) { counts[0] += m; }

// Host snapshots and ring slots are planar, unpadded (u, v[, w] planes of the storage type,
// round to nearest even): 25% fewer bytes per 3D upload than padded nodes.
template <typename T>
__device__ __forceinline__ T to_storage(float x) {
    if constexpr (std::is_same<T, __nv_bfloat16>::value) return __float2bfloat16_rn(x);
    else if constexpr (std::is_same<T, __half>::value) return __float2half_rn(x);
    else return x;
}

template <typename T>
__global__ void planar_pack_kernel(const float *__restrict__ u, const float *__restrict__ v,
                                   const float *__restrict__ w, T *__restrict__ out, int64_t nodes, int dim) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        out[i] = to_storage<T>(u[i]);
        out[nodes + i] = to_storage<T>(v[i]);
        if (dim == 3) out[2 * nodes + i] = to_storage<T>(w[i]);
    }
}

// Two planar slots -> the window-pair layout the step kernel reads (granite_kernels.cuh,
// Store<Pair<...>>): per node, component by component, back then front: {u_b, u_f, v_b, v_f,
// w_b, w_f, 0, 0} (3D) or {u_b, u_f, v_b, v_f} (2D), vector stores.  3D pairs carry the zero
// border of pair_pack_padded_kernel (pack_kernels.cuh): every padded node (nx + 3) x (ny + 3) x
// (nz + 3) is written, zeros outside the grid; 2D pairs replicate the edge nodes.
template <typename T>
__global__ void planar_pair_kernel(const T *__restrict__ b, const T *__restrict__ f, T *__restrict__ out,
                                   int64_t nodes, int dim, int32_t nx, int32_t ny, int32_t nz) {
    using V = typename std::conditional<sizeof(T) == 4, uint4, uint2>::type;   // 4 values of T
    if (dim == 3) {
        const int32_t pnx = nx + 3, pny = ny + 3;
        const int32_t total = pnx * pny * (nz + 3);
        for (int32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
            const int32_t x = o % pnx - 1, r = o / pnx;
            const int32_t y = r % pny - 1, z = r / pny - 1;
            const T zero = to_storage<T>(0.f);
            alignas(sizeof(V)) T lo[4] = {zero, zero, zero, zero};
            alignas(sizeof(V)) T hi[4] = {zero, zero, zero, zero};
            if ((unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz) {
                const int64_t i = ((int64_t)z * ny + y) * nx + x;
                lo[0] = b[i]; lo[1] = f[i]; lo[2] = b[nodes + i]; lo[3] = f[nodes + i];
                hi[0] = b[2 * nodes + i]; hi[1] = f[2 * nodes + i];
            }
            V *po = reinterpret_cast<V *>(out + 8 * (int64_t)o);
            po[0] = *reinterpret_cast<const V *>(lo);
            po[1] = *reinterpret_cast<const V *>(hi);
        }
        return;
    }
    // 2D: replicated edges (pair_pack_edge2_kernel, pack_kernels.cuh)
    const int32_t pnx = nx + 3;
    const int32_t total = pnx * (ny + 3);
    for (int32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
        const int32_t x = min(max(o % pnx - 1, 0), nx - 1), y = min(max(o / pnx - 1, 0), ny - 1);
        const int64_t i = (int64_t)y * nx + x;
        alignas(sizeof(V)) T q[4] = {b[i], f[i], b[nodes + i], f[nodes + i]};
        *reinterpret_cast<V *>(out + 4 * (int64_t)o) = *reinterpret_cast<const V *>(q);
    }
}

__global__ void init_pool_kernel(int32_t *counts) {
    counts[0] = 0;
    counts[1] = 0;
    counts[2] = 0;
    counts[3] = 0;
}

int setup(gr_server *S, int64_t nz, int64_t ny, int64_t nx) {
    S->nx = nx; S->ny = ny; S->nz = S->dim == 3 ? nz : 1;
    S->nodes = S->nx * S->ny * S->nz;
    const gr_settings &s = S->s;
    const float *gs = s.grid_scale, *of = s.offset;
    if (s.grid_scale_len == 1) { S->scale[0] = S->scale[1] = S->scale[2] = gs[0]; }
    else if (s.grid_scale_len == 2) { S->scale[0] = gs[0]; S->scale[1] = gs[1]; S->scale[2] = gs[0]; }
    else if (s.grid_scale_len == 3) { S->scale[0] = gs[0]; S->scale[1] = gs[1]; S->scale[2] = gs[2]; }
    else return SUSER("Invalid GridScale dimension.");
    if (s.offset_len == 1) { S->off[0] = S->off[1] = S->off[2] = of[0]; }
    else if (s.grid_scale_len == 2 && s.offset_len >= 2) { S->off[0] = of[0]; S->off[1] = of[1]; S->off[2] = of[0]; }
    else if (s.grid_scale_len == 3 && s.offset_len >= 3) { S->off[0] = of[0]; S->off[1] = of[1]; S->off[2] = of[2]; }
    else return SUSER("Invalid Offset dimension.");
    const float g[3] = {(float)S->nx, (float)S->ny, (float)(S->dim == 3 ? nz : 0)};
    for (int d = 0; d < 3; ++d) {
        S->dom[d] = g[d] * S->scale[d];
        S->inv_scale[d] = 1.0f / S->scale[d];
    }
    S->elem = s.storage == GR_STORE_F32 ? 4 : 2;
    S->snap_bytes = S->nodes * S->dim * S->elem;                  // planar, unpadded
    S->slot_stride = ((S->snap_bytes + 255) / 256) * 256;
    SK(S->ring.alloc((size_t)S->slot_stride * kRing));
    // window pairs carry a border (padded_pair_nodes); the kernel indexes them with int32
    if (padded_pair_nodes(S->dim, S->nx, S->ny, S->nz) > (int64_t(1) << 31) - 1)
        return SUSER("Invalid dataset was provided. Grid too large.");
    SK(S->pair.alloc((size_t)padded_pair_nodes(S->dim, S->nx, S->ny, S->nz) * (S->dim == 3 ? 8 : 4) * S->elem));
    SK(S->raw.alloc((size_t)S->nodes * S->dim));
    S->host_snap.assign((size_t)S->n_snap, nullptr);
    for (int k = 0; k < kRing; ++k) S->ring_holds[k] = -1;
    // Morton-ranked bricks for the pools' spatial sort (as in the engine)
    S->bx = 4; S->by = 4; S->bz = S->dim == 3 ? 2 : 1;
    for (;;) {
        S->nbx = (int)((S->nx + S->bx - 1) / S->bx);
        S->nby = (int)((S->ny + S->by - 1) / S->by);
        S->nbz = (int)((S->nz + S->bz - 1) / S->bz);
        if ((int64_t)S->nbx * S->nby * S->nbz <= (1 << 20) && S->nbx <= 1024 && S->nby <= 1024 && S->nbz <= 1024) break;
        S->bx *= 2; S->by *= 2; if (S->dim == 3) S->bz *= 2;
    }
    S->nbins = S->nbx * S->nby * S->nbz;
    auto spread = [](uint32_t v) {
        uint64_t x = v & 0x3ff;
        x = (x | (x << 16)) & 0x030000FF;
        x = (x | (x << 8)) & 0x0300F00F;
        x = (x | (x << 4)) & 0x030C30C3;
        x = (x | (x << 2)) & 0x09249249;
        return x;
    };
    std::vector<std::pair<uint64_t, int32_t>> codes((size_t)S->nbins);
    for (int z = 0; z < S->nbz; ++z)
        for (int y = 0; y < S->nby; ++y)
            for (int x = 0; x < S->nbx; ++x) {
                const int32_t lin = (z * S->nby + y) * S->nbx + x;
                codes[lin] = {spread(x) | (spread(y) << 1) | (spread(z) << 2), lin};
            }
    std::sort(codes.begin(), codes.end());
    std::vector<int32_t> tab((size_t)S->nbins);
    for (int32_t r = 0; r < S->nbins; ++r) tab[codes[r].second] = r;
    SK(S->bintab.alloc(tab.size()));
    SK(cudaMemcpy(S->bintab.p, tab.data(), tab.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    SK(S->hist.alloc((size_t)S->nbins + 1));
    SK(S->chunk.alloc((size_t)(S->nbins + 1 + SCAN_CHUNK - 1) / SCAN_CHUNK));
    return GR_OK;
}

// Pools, result arena and staging sized from the HBM budget.
int allocate(gr_server *S, int64_t budget) {
    // per pool slot: 7 arrays x 2 buffers + key + perm = 64 bytes; per arena slot 16 bytes
    const int64_t per = 2 * 64 + 2 * 16;
    int64_t cap = budget / per;
    cap = std::min<int64_t>(cap, (int64_t(1) << 31) / 2 - 1);
    if (cap < 1024) return SUSER("HBM budget too small for the request server.");
    for (int p = 0; p < 2; ++p) {
        Pool &P = S->pools[p];
        P.cap = cap;
        for (auto &a : P.st) {
            SK(a.px.alloc(cap)); SK(a.py.alloc(cap));
            if (S->dim == 3) SK(a.pz.alloc(cap));
            SK(a.status.alloc(cap)); SK(a.id.alloc(cap)); SK(a.life.alloc(cap)); SK(a.birth.alloc(cap));
        }
        SK(P.key.alloc(cap));
        SK(P.perm.alloc(cap));
        SK(P.counts.alloc(4));
        init_pool_kernel<<<1, 1, 0, S->cs>>>(P.counts.p);
        SK(cudaGetLastError());
        P.threads = 256;
        const int st = S->s.storage;
        // positions only (no curvature, volumes, constants, uplift, length abort, compensation):
        // the lean variant unless 2D loop borders, sphere coordinates or 1/256 filter weights are on
        const bool lean = !(S->dim == 2 && (S->s.border_mode != 0 || S->s.sphere_radius > 0.f)) &&
                          !S->s.filter_weights;
        const int ft = lean ? FT_LEAN : FT_GENERIC;
        P.fn = st == GR_STORE_BF16 ? advance_bf16(S->dim, p == 1, true, ft)
             : st == GR_STORE_F16 ? advance_f16(S->dim, p == 1, true, ft) : advance_f32(S->dim, p == 1, true, ft);
        cudaFuncAttributes fa{};
        SK(cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(P.fn)));
        P.threads = std::min(P.threads, fa.maxThreadsPerBlock);   // the kernel's launch bounds
        int per_sm = 0, sms = 0;
        SK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, P.fn, P.threads, 0));
        SK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, S->s.device));
        P.grid = (int64_t)std::max(1, per_sm) * sms;
    }
    S->arena_cap = 2 * cap;
    SK(S->res_px.alloc(S->arena_cap)); SK(S->res_py.alloc(S->arena_cap));
    if (S->dim == 3) SK(S->res_pz.alloc(S->arena_cap));
    SK(S->res_status.alloc(S->arena_cap));
    S->arena.reset(S->arena_cap);
    SK(S->counters.alloc(4));
    SK(cudaMemsetAsync(S->counters.p, 0, 4 * sizeof(unsigned long long), S->cs));
    S->st.capacity_particles = cap;
    return GR_OK;
}

KParams pool_params(gr_server *S, Pool &P) {
    KParams K;
    std::memset(&K, 0, sizeof K);
    for (int d = 0; d < 3; ++d) {
        K.inv_scale[d] = S->inv_scale[d];
        K.off[d] = S->off[d];
        K.dom[d] = S->dom[d];
        K.scale[d] = S->scale[d];
    }
    K.nx = (int32_t)S->nx; K.ny = (int32_t)S->ny; K.nz = (int32_t)S->nz; K.dim = S->dim;
    K.fn[0] = (float)S->nx; K.fn[1] = (float)S->ny; K.fn[2] = (float)S->nz;
    K.wind = S->ring.p;
    K.wind_stride = S->slot_stride;
    K.pair = S->pair.p;
    K.pnx = (int32_t)(S->nx + 3); K.pnxy = (int32_t)((S->nx + 3) * (S->ny + 3));
    Pool::Arrays &A = P.st[P.cur];
    K.px = A.px.p; K.py = A.py.p; K.pz = A.pz.p;
    K.status = A.status.p; K.id = A.id.p; K.life = A.life.p; K.birth = A.birth.p;
    K.n = P.cap; K.n_state = P.cap; K.n_total = P.cap;
    K.n_dev = P.counts.p;
    K.grid_stride = 1;
    K.sched = S->d_sched.p;
    const gr_settings &s = S->s;
    K.h = s.delta_t;
    K.hh = 0.5f * s.delta_t;
    K.sixth = 1.0f / 6;
    K.inv_2h = 1.0f / (2.0f * s.delta_t);
    K.inv_hh = 1.0f / (s.delta_t * s.delta_t);
    K.sphere_radius = s.sphere_radius;
    K.wind_dynamic = 1;
    K.dyn_any = 1;
    K.border_mode = S->dim == 2 ? s.border_mode : 0;
    K.reverse = s.reverse ? 1 : 0;
    K.sphere = S->dim == 2 && s.sphere_radius > 0.f;
    K.filter_weights = s.filter_weights ? 1 : 0;
    K.counters = S->counters.p;
    return K;
}

StateView pool_view(Pool::Arrays &A) {
    StateView v;
    std::memset(&v, 0, sizeof v);
    v.px = A.px.p; v.py = A.py.p; v.pz = A.pz.p;
    v.status = A.status.p; v.id = A.id.p; v.life = A.life.p; v.birth = A.birth.p;
    return v;
}

int compact_pool(gr_server *S, Pool &P, int32_t k_end) {
    CompactParams C;
    std::memset(&C, 0, sizeof C);
    C.src = pool_view(P.st[P.cur]);
    C.dst = pool_view(P.st[1 - P.cur]);
    StateView R;
    std::memset(&R, 0, sizeof R);
    R.px = S->res_px.p; R.py = S->res_py.p; R.pz = S->res_pz.p; R.status = S->res_status.p;
    C.ret = R;
    C.ret_by_id = 1;
    C.key = P.key.p;
    C.hist = S->hist.p;
    C.chunk = S->chunk.p;
    C.perm = P.perm.p;
    C.bintab = S->bintab.p;
    C.n_act = P.counts.p;
    C.n_new = P.counts.p + 1;
    C.n_ret = P.counts.p + 2;
    for (int d = 0; d < 3; ++d) {
        C.off[d] = S->off[d];
        C.inv_scale[d] = S->inv_scale[d];
    }
    C.nx = (int32_t)S->nx; C.ny = (int32_t)S->ny; C.nz = (int32_t)S->nz; C.dim = S->dim;
    C.bx = S->bx; C.by = S->by; C.bz = S->bz; C.nbx = S->nbx; C.nby = S->nby; C.nbz = S->nbz; C.nbins = S->nbins;
    C.k_end = k_end;
    const int threads = 256;
    const int blocks = std::min(grid_for(std::max<int64_t>(1, P.in_flight), threads), 148 * 16);
    // retired particles go to their result slots: the retired count is not needed
    SK(cudaMemsetAsync(P.counts.p + 2, 0, sizeof(int32_t), S->cs));
    const int nchunks = (S->nbins + 1 + SCAN_CHUNK - 1) / SCAN_CHUNK;
    SK(cudaMemsetAsync(S->hist.p, 0, ((size_t)S->nbins + 1) * sizeof(int32_t), S->cs));
    bin_kernel<<<blocks, threads, 0, S->cs>>>(C);
    scan_chunks_kernel<<<nchunks, SCAN_CHUNK, 0, S->cs>>>(C);
    scan_top_kernel<<<1, 1024, 0, S->cs>>>(C, nchunks);
    rank_kernel<<<blocks, threads, 0, S->cs>>>(C);
    gather_kernel<<<blocks, threads, 0, S->cs>>>(C);
    commit_kernel<<<1, 1, 0, S->cs>>>(C);
    SK(cudaGetLastError());
    P.cur = 1 - P.cur;
    return GR_OK;
}

// Virtual snapshot v (sweep * n_snap + snapshot) resident in slot v % kRing, loaded on the
// copy stream once the slot's previous window is done.
int ensure_snapshot(gr_server *S, int64_t v) {
    const int slot = (int)(v % kRing);
    if (S->ring_holds[slot] == v) return GR_OK;
    const int64_t snap = v % S->n_snap;
    if (S->slot_used[slot]) SK(cudaStreamWaitEvent(S->xs, S->slot_free[slot], 0));
    SK(cudaMemcpyAsync(S->ring.p + (int64_t)slot * S->slot_stride, S->host_snap[snap], (size_t)S->snap_bytes,
                       cudaMemcpyHostToDevice, S->xs));
    SK(cudaEventRecord(S->slot_ready[slot], S->xs));
    S->ring_holds[slot] = v;
    S->st.h2d_bytes += S->snap_bytes;
    return GR_OK;
}

int pack_pair(gr_server *S, int64_t v) {
    const char *back = S->ring.p + (v % kRing) * S->slot_stride;
    const char *front = S->ring.p + ((v + 1) % kRing) * S->slot_stride;
    const int threads = 256, blocks = grid_for(S->nodes, threads);
    switch (S->s.storage) {
        case GR_STORE_BF16:
            planar_pair_kernel<__nv_bfloat16><<<blocks, threads, 0, S->cs>>>(
                (const __nv_bfloat16 *)back, (const __nv_bfloat16 *)front, (__nv_bfloat16 *)S->pair.p, S->nodes, S->dim,
                (int32_t)S->nx, (int32_t)S->ny, (int32_t)S->nz);
            break;
        case GR_STORE_F16:
            planar_pair_kernel<__half><<<blocks, threads, 0, S->cs>>>((const __half *)back, (const __half *)front,
                                                                     (__half *)S->pair.p, S->nodes, S->dim,
                                                                     (int32_t)S->nx, (int32_t)S->ny, (int32_t)S->nz);
            break;
        default:
            planar_pair_kernel<float><<<blocks, threads, 0, S->cs>>>((const float *)back, (const float *)front,
                                                                    (float *)S->pair.p, S->nodes, S->dim,
                                                                    (int32_t)S->nx, (int32_t)S->ny, (int32_t)S->nz);
            break;
    }
    SK(cudaGetLastError());
    return GR_OK;
}

// Requests admitted in this window -> device staging -> their pool's tail.
int admit(gr_server *S, const std::vector<Req *> &adm) {
    for (int p = 0; p < 2; ++p) {
        int64_t m = 0;
        for (Req *r : adm)
            if (r->integrator == p) m += r->n;
        if (m == 0) continue;
        gr_server::Stage &G = S->stage[S->stage_next];
        S->stage_next ^= 1;
        if (G.ev) SK(cudaEventSynchronize(G.ev));   // its previous upload has been read
        else SK(cudaEventCreateWithFlags(&G.ev, cudaEventDisableTiming));
        if (m > G.cap) {
            if (G.h) SK(cudaFreeHost(G.h));
            G.h = nullptr;
            const int64_t cap = std::max<int64_t>(m, 1 << 20);
            SK(cudaMallocHost(&G.h, (size_t)cap * (S->dim + 3) * sizeof(float)));
            G.cap = cap;
            SK(G.seeds.alloc((size_t)cap * S->dim));
            SK(G.meta.alloc((size_t)cap * 3));
        }
        int32_t *meta = reinterpret_cast<int32_t *>(G.h + m * S->dim);
        int64_t o = 0;
        for (Req *r : adm) {
            if (r->integrator != p) continue;
            std::memcpy(G.h + o * S->dim, r->seeds.data(), (size_t)r->n * S->dim * sizeof(float));
            for (int64_t i = 0; i < r->n; ++i) {
                meta[o + i] = (int32_t)(r->slot + i);
                meta[m + o + i] = (int32_t)r->end_step;
                meta[2 * m + o + i] = (int32_t)r->start_step;
            }
            o += r->n;
            std::vector<float>().swap(r->seeds);
        }
        SK(cudaMemcpyAsync(G.seeds.p, G.h, (size_t)m * S->dim * sizeof(float), cudaMemcpyHostToDevice, S->cs));
        SK(cudaMemcpyAsync(G.meta.p, meta, (size_t)m * 3 * sizeof(int32_t), cudaMemcpyHostToDevice, S->cs));
        SK(cudaEventRecord(G.ev, S->cs));
        Pool &P = S->pools[p];
        Pool::Arrays &A = P.st[P.cur];
        append_kernel<<<grid_for(m, 256), 256, 0, S->cs>>>(G.seeds.p, G.meta.p, m, S->dim, P.counts.p, A.px.p,
                                                           A.py.p, A.pz.p, A.status.p, A.id.p, A.life.p, A.birth.p);
        grow_kernel<<<1, 1, 0, S->cs>>>(P.counts.p, (int32_t)m);
        SK(cudaGetLastError());
        P.in_flight += m;
        S->st.h2d_bytes += m * (S->dim * 4 + 12);
    }
    return GR_OK;
}

// One window of the sweep; returns the requests that complete in it.
int run_window(gr_server *S, const std::vector<Req *> &adm, const std::vector<Req *> &finishing) {
    const int64_t v = S->sweep * S->n_snap + S->w;
    // keep at most kLag windows in flight
    cudaEvent_t lag = S->win_done[S->win_count % S->win_done.size()];
    if (S->win_count >= (int64_t)S->win_done.size()) SK(cudaEventSynchronize(lag));
    for (int64_t k = v; k < v + kRing && k < (S->sweep + 1) * S->n_snap; ++k) {
        const int slot = (int)(k % kRing);
        if (k >= v + 2 && S->slot_used[slot] && S->ring_holds[slot] != k) {
            // prefetch only into slots whose previous use has finished
            if (cudaEventQuery(S->slot_free[slot]) != cudaSuccess) break;
        }
        const int rc = ensure_snapshot(S, k);
        if (rc) return rc;
    }
    SK(cudaStreamWaitEvent(S->cs, S->slot_ready[v % kRing], 0));
    SK(cudaStreamWaitEvent(S->cs, S->slot_ready[(v + 1) % kRing], 0));
    int rc = admit(S, adm);
    if (rc) return rc;
    const int64_t k0 = S->sched.window_begin[S->w], k1 = S->sched.window_begin[S->w + 1];
    const bool any = S->pools[0].in_flight > 0 || S->pools[1].in_flight > 0;
    if (any) {
        rc = pack_pair(S, v);
        if (rc) return rc;
    }
    for (int p = 0; p < 2; ++p) {
        Pool &P = S->pools[p];
        if (P.in_flight == 0) continue;
        KParams K = pool_params(S, P);
        K.s0 = (int32_t)k0;
        K.s1 = (int32_t)k1;
        P.fn<<<(unsigned)P.grid, P.threads, 0, S->cs>>>(K);
        SK(cudaGetLastError());
        rc = compact_pool(S, P, (int32_t)k1);
        if (rc) return rc;
    }
    for (int k = 0; k < 2; ++k) {
        const int slot = (int)((v + k) % kRing);
        SK(cudaEventRecord(S->slot_free[slot], S->cs));
        S->slot_used[slot] = true;
    }
    // results of the requests that end in this window
    for (Req *r : finishing) {
        const int64_t n = r->n, D = S->dim;
        float *dst = S->pin_res + r->stage;
        SK(cudaMemcpyAsync(dst, S->res_px.p + r->slot, n * 4, cudaMemcpyDeviceToHost, S->cs));
        SK(cudaMemcpyAsync(dst + n, S->res_py.p + r->slot, n * 4, cudaMemcpyDeviceToHost, S->cs));
        if (D == 3) SK(cudaMemcpyAsync(dst + 2 * n, S->res_pz.p + r->slot, n * 4, cudaMemcpyDeviceToHost, S->cs));
        SK(cudaMemcpyAsync(dst + D * n, S->res_status.p + r->slot, n * 4, cudaMemcpyDeviceToHost, S->cs));
        if (!r->done_ev) SK(cudaEventCreateWithFlags(&r->done_ev, cudaEventDisableTiming));
        SK(cudaEventRecord(r->done_ev, S->cs));
        S->pools[r->integrator].in_flight -= n;
        S->st.d2h_bytes += n * (D + 1) * 4;
    }
    SK(cudaEventRecord(lag, S->cs));
    ++S->win_count;
    ++S->st.windows;
    return GR_OK;
}

// Hands out the results whose copies have finished (worker thread, lock held).
void collect(gr_server *S, bool block) {
    for (size_t k = 0; k < S->returning.size();) {
        Req *r = S->reqs[S->returning[k]].get();
            cudaError_t q = block && k == 0 ? cudaEventSynchronize(r->done_ev) : cudaEventQuery(r->done_ev);
        if (q == cudaErrorNotReady) {
            ++k;
            continue;
        }
        if (q != cudaSuccess && S->failure.empty()) S->failure = cudaGetErrorString(q);
        const int64_t n = r->n, D = S->dim;
        const float *src = S->pin_res + r->stage;
        r->pos.resize((size_t)n * D);
        r->status.resize((size_t)n);
        for (int64_t i = 0; i < n; ++i)
            for (int64_t d = 0; d < D; ++d) r->pos[i * D + d] = src[d * n + i];
        std::memcpy(r->status.data(), src + D * n, (size_t)n * 4);
        S->pin_alloc.give(r->stage, n * (D + 1));
        S->arena.give(r->slot, n);
        r->state = r->cancelled ? GR_REQ_CANCELLED : GR_REQ_DONE;
        r->t_done = S->now();
        if (r->cancelled) {
            std::vector<float>().swap(r->pos);
            std::vector<int32_t>().swap(r->status);
        }
        ++S->st.completed;
        S->returning.erase(S->returning.begin() + (long)k);
    }
    S->done_cv.notify_all();
}

void work(gr_server *S) {
    cudaSetDevice(S->s.device);
    std::unique_lock<std::mutex> lk(S->mu);
    for (;;) {
        S->cv.wait(lk, [&] {
            return S->stop || !S->pending.empty() || !S->active.empty() || !S->returning.empty();
        });
        if (S->stop) break;
        if (S->active.empty() && S->pending.empty()) {
            // nothing left to integrate: wait for the oldest result copy
            cudaEvent_t ev = S->reqs[S->returning.front()]->done_ev;
            lk.unlock();
            cudaEventSynchronize(ev);
            lk.lock();
            collect(S, false);
            continue;
        }
        if (S->active.empty()) {
            // empty pools: jump to the earliest start window still ahead in this sweep, else
            // to the earliest one in the next sweep
            int64_t ahead = -1, first = -1;
            for (int64_t id : S->pending) {
                const int64_t sw = S->reqs[id]->start_window;
                if (sw >= S->w && (ahead < 0 || sw < ahead)) ahead = sw;
                if (first < 0 || sw < first) first = sw;
            }
            if (ahead >= 0 && ahead != S->w) {
                S->w = ahead;
                ++S->st.jumps;
            } else if (ahead < 0) {
                S->w = first;
                ++S->sweep;
                ++S->st.sweeps;
                ++S->st.jumps;
            }
        }
        // admission in arrival order; a request that does not fit waits (a later, smaller one
        // may still enter)
        std::vector<Req *> adm;
        for (auto it = S->pending.begin(); it != S->pending.end();) {
            Req *r = S->reqs[*it].get();
            if (r->start_window != S->w) {
                ++it;
                continue;
            }
            Pool &P = S->pools[r->integrator];
            int64_t admitted_here = 0;
            for (Req *a : adm)
                if (a->integrator == r->integrator) admitted_here += a->n;
            if (P.in_flight + admitted_here + r->n > P.cap) {
                ++S->st.deferred;
                ++it;
                continue;
            }
            const int64_t slot = S->arena.take(r->n);
            if (slot < 0) {
                ++S->st.deferred;
                ++it;
                continue;
            }
            r->slot = slot;
            r->state = GR_REQ_ACTIVE;
            r->t_admit = S->now();
            adm.push_back(r);
            S->active.push_back(r->id);
            ++S->st.admitted;
            it = S->pending.erase(it);
        }
        int64_t inflight = S->pools[0].in_flight + S->pools[1].in_flight;
        for (Req *a : adm) inflight += a->n;
        S->st.peak_particles = std::max(S->st.peak_particles, inflight);
        const int64_t k1 = S->sched.window_begin[S->w + 1];
        std::vector<Req *> fin;
        for (size_t k = 0; k < S->active.size();) {
            Req *r = S->reqs[S->active[k]].get();
            if (r->ended || r->end_step <= k1) {
                r->ended = true;
                // pinned room for its results; wait for earlier copies to drain if needed.  When
                // this window's own completions fill the staging, the rest stay in the result
                // arena and are copied in a later window.
                int64_t stage;
                while ((stage = S->pin_alloc.take(r->n * (S->dim + 1))) < 0 && !S->returning.empty()) {
                    cudaEvent_t ev = S->reqs[S->returning.front()]->done_ev;
                    lk.unlock();
                    cudaEventSynchronize(ev);
                    lk.lock();
                    collect(S, false);
                }
                if (stage < 0) {
                    ++S->st.staged_later;
                    ++k;
                    continue;
                }
                r->stage = stage;
                fin.push_back(r);
                S->active.erase(S->active.begin() + (long)k);
            } else {
                ++k;
            }
        }
        int rc = S->failure.empty() ? GR_OK : GR_ERR_RUNTIME;
        if (!rc) {
            lk.unlock();
            rc = run_window(S, adm, fin);
            lk.lock();
        }
        // their result copies are enqueued now: collect() may wait for them
        for (Req *r : fin) S->returning.push_back(r->id);
        if (rc) {
            if (S->failure.empty()) S->failure = gr_last_error();
            for (auto &kv : S->reqs)
                if (kv.second->state == GR_REQ_PENDING || kv.second->state == GR_REQ_ACTIVE)
                    kv.second->state = GR_REQ_FAILED;
            S->pending.clear();
            S->active.clear();
            S->returning.clear();
            S->done_cv.notify_all();
            break;
        }
        collect(S, false);
        if (++S->w >= S->W) {
            S->w = 0;
            ++S->sweep;
            ++S->st.sweeps;
        }
    }
}

}  // namespace

gr_server::~gr_server() {
    {
        std::lock_guard<std::mutex> g(mu);
        stop = true;
    }
    cv.notify_all();
    if (worker.joinable()) worker.join();
    if (cs) cudaStreamSynchronize(cs);
    if (xs) cudaStreamSynchronize(xs);
    for (auto &kv : reqs)
        if (kv.second->done_ev) cudaEventDestroy(kv.second->done_ev);
    for (void *p : host_snap)
        if (p) cudaFreeHost(p);
    if (pin_res) cudaFreeHost(pin_res);
    for (auto &g : stage) {
        if (g.h) cudaFreeHost(g.h);
        if (g.ev) cudaEventDestroy(g.ev);
    }
    for (int k = 0; k < kRing; ++k) {
        if (slot_ready[k]) cudaEventDestroy(slot_ready[k]);
        if (slot_free[k]) cudaEventDestroy(slot_free[k]);
    }
    for (auto e : win_done) cudaEventDestroy(e);
    if (cs) cudaStreamDestroy(cs);
    if (xs) cudaStreamDestroy(xs);
}

extern "C" {

int gr_server_create(const gr_settings *settings, int64_t n_snapshots, int64_t nz, int64_t ny, int64_t nx,
                     int64_t hbm_budget_bytes, gr_server **out) {
    if (!settings || !out) return SUSER("null argument");
    *out = nullptr;
    const gr_settings &s = *settings;
    if (s.space != 0 && s.space != 1) return SUSER("Invalid Space.");
    if (s.windfield_mode != 1) return SUSER("The request server needs a Dynamic windfield.");
    if (s.curvature_mode != 0 || s.volume_mode != 0 || s.constants_mode != 0 || s.uplift_mode != 0 ||
        s.abort_mode != 0 || s.minimum_alive != 0 || s.compensated != 0)
        return SUSER("The request server integrates positions only (no curvature, volumes, constants, uplift, "
                     "length abort, MinimumAliveParticles or compensation).");
    if (s.delta_t <= 0.f || !std::isfinite(s.delta_t)) return SUSER("DeltaT must be positive.");
    if (s.data_time_distance <= 0.f || !std::isfinite(s.data_time_distance)) return SUSER("DataTimeDistance must be positive.");
    if (s.storage < 0 || s.storage > 2) return SUSER("Invalid storage type.");
    if (n_snapshots < 2) return SUSER("The field needs at least two snapshots.");
    if (nx < 1 || ny < 1 || nz < 1 || nx > (1 << 30) || ny > (1 << 30) || nz > (1 << 30))
        return SUSER("Invalid dataset was provided. Empty grid.");
    auto S = std::make_unique<gr_server>();
    S->s = s;
    S->dim = s.space == 0 ? 3 : 2;
    S->n_snap = n_snapshots;
    SK(cudaSetDevice(s.device));
    SK(cudaStreamCreateWithFlags(&S->cs, cudaStreamNonBlocking));
    SK(cudaStreamCreateWithFlags(&S->xs, cudaStreamNonBlocking));
    for (int k = 0; k < kRing; ++k) {
        SK(cudaEventCreateWithFlags(&S->slot_ready[k], cudaEventDisableTiming));
        SK(cudaEventCreateWithFlags(&S->slot_free[k], cudaEventDisableTiming));
    }
    S->win_done.assign(kLag + 1, nullptr);
    for (auto &e : S->win_done) SK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    int rc = setup(S.get(), S->dim == 3 ? nz : 1, ny, nx);
    if (rc) return rc;
    // the field's global step clock: the reference's float32 schedule over all windows
    ScheduleInput si;
    si.dyn_any = true;
    si.wind_dynamic = true;
    si.delta_t = s.delta_t;
    si.data_time_distance = s.data_time_distance;
    si.maximum_simulation_time = (float)(n_snapshots - 1) * s.data_time_distance;
    si.save_interval = 0;
    si.time_mode = s.time_mode;
    S->sched = build_schedule(si);
    if ((int64_t)S->sched.window_begin.size() - 1 > n_snapshots - 1) {
        S->sched.window_begin.resize((size_t)n_snapshots);
        S->sched.steps.resize((size_t)S->sched.window_begin.back());
    }
    S->W = (int64_t)S->sched.window_begin.size() - 1;
    if (S->W < 1 || S->sched.steps.empty()) return SUSER("The field window holds no integration step.");
    std::vector<StepEntry> hs(S->sched.steps.size());
    for (size_t k = 0; k < hs.size(); ++k) {
        const HostStep &h = S->sched.steps[k];
        StepEntry E{};
        E.t0 = h.t0; E.t1 = h.t1; E.t2 = h.t2;
        E.flags = h.time_pos ? SF_TIME_POS : 0;
        hs[k] = E;
    }
    SK(S->d_sched.alloc(hs.size()));
    SK(cudaMemcpy(S->d_sched.p, hs.data(), hs.size() * sizeof(StepEntry), cudaMemcpyHostToDevice));
    int64_t budget = hbm_budget_bytes;
    if (budget <= 0) {
        size_t fr = 0, tot = 0;
        SK(cudaMemGetInfo(&fr, &tot));
        budget = (int64_t)((fr + dev_pool_idle_bytes()) / 4);   // the pool's idle memory is ours to use
    }
    rc = allocate(S.get(), budget);
    if (rc) return rc;
    // pinned result staging: a quarter of the arena (at most 256 MB), never less than one full
    // pool, so any admissible request fits; completions beyond it wait a window
    S->pin_res_cap = std::max<int64_t>(std::min<int64_t>(S->arena_cap * (S->dim + 1) / 4, int64_t(64) << 20),
                                       S->pools[0].cap * (S->dim + 1));
    SK(cudaMallocHost(&S->pin_res, (size_t)S->pin_res_cap * sizeof(float)));
    S->pin_alloc.reset(S->pin_res_cap);
    SK(cudaStreamSynchronize(S->cs));
    *out = S.release();
    return GR_OK;
}

int gr_server_set_snapshot(gr_server *S, int64_t snapshot, const float *const *comps, int32_t ncomp,
                           int32_t device_src) {
    if (!S) return SUSER("null server");
    if (S->started) return SUSER("Snapshots are fixed once the server has started.");
    if (snapshot < 0 || snapshot >= S->n_snap) return SUSER("snapshot index out of range");
    if (ncomp != S->dim || !comps) return SUSER("Invalid dataset was provided. Wrong amount of data.");
    for (int c = 0; c < ncomp; ++c)
        if (!comps[c]) return SUSER("null windfield component");
    SK(cudaSetDevice(S->s.device));
    const size_t plane = (size_t)S->nodes;
    const float *src[3];
    for (int c = 0; c < ncomp; ++c) {
        if (device_src) {
            src[c] = comps[c];
        } else {
            SK(cudaMemcpy(S->raw.p + c * plane, comps[c], plane * sizeof(float), cudaMemcpyHostToDevice));
            src[c] = S->raw.p + c * plane;
        }
    }
    if (ncomp == 2) src[2] = src[1];
    char *scratch = S->ring.p;   // slot 0 as packing scratch before the server starts
    const int threads = 256, blocks = grid_for(S->nodes, threads);
    switch (S->s.storage) {
        case GR_STORE_BF16:
            planar_pack_kernel<__nv_bfloat16><<<blocks, threads, 0, S->cs>>>(src[0], src[1], src[2], (__nv_bfloat16 *)scratch,
                                                                             S->nodes, S->dim);
            break;
        case GR_STORE_F16:
            planar_pack_kernel<__half><<<blocks, threads, 0, S->cs>>>(src[0], src[1], src[2], (__half *)scratch, S->nodes, S->dim);
            break;
        default:
            planar_pack_kernel<float><<<blocks, threads, 0, S->cs>>>(src[0], src[1], src[2], (float *)scratch, S->nodes, S->dim);
            break;
    }
    SK(cudaGetLastError());
    void *&h = S->host_snap[(size_t)snapshot];
    if (!h) SK(cudaMallocHost(&h, (size_t)S->snap_bytes));
    SK(cudaMemcpyAsync(h, scratch, (size_t)S->snap_bytes, cudaMemcpyDeviceToHost, S->cs));
    SK(cudaStreamSynchronize(S->cs));
    return GR_OK;
}

int gr_server_start(gr_server *S) {
    if (!S) return SUSER("null server");
    if (S->started) return GR_OK;
    for (void *p : S->host_snap)
        if (!p) return SUSER("Every snapshot must be set before the server starts.");
    for (int k = 0; k < kRing; ++k) S->ring_holds[k] = -1;
    S->started = true;
    S->t0 = std::chrono::steady_clock::now();
    S->worker = std::thread(work, S);
    return GR_OK;
}

int gr_server_submit(gr_server *S, const float *seeds, int64_t n, int32_t dim, double start_time, int32_t steps,
                     int32_t integrator, int64_t *id) {
    if (!S || !id) return SUSER("null argument");
    if (!S->started) return SUSER("The server has not started.");
    if (dim != S->dim) return SUSER("Dimensions of IntegratorSettings and provided TrajectorySet do not match.");
    if (n <= 0 || !seeds) return SUSER("Provided TrajectorySet does not contain any data.");
    if (integrator != 0 && integrator != 1) return SUSER("Invalid Integrator.");
    if (steps < 0) return SUSER("steps must not be negative");
    const int64_t total = (int64_t)S->sched.steps.size();
    // the step that contains the start time
    int64_t k0 = (int64_t)std::floor(start_time / (double)S->s.delta_t + 1e-9);
    if (k0 < 0 || k0 >= total) return SUSER("start time outside the field window");
    auto r = std::make_unique<Req>();
    r->integrator = integrator;
    r->n = n;
    r->start_step = k0;
    r->end_step = std::min<int64_t>(total, k0 + steps);
    r->start_window = S->sched.steps[(size_t)k0].window;
    if (r->end_step <= k0) r->end_step = k0;
    r->seeds.assign(seeds, seeds + n * dim);
    std::lock_guard<std::mutex> g(S->mu);
    if (!S->failure.empty()) return sfail(GR_ERR_RUNTIME, "ERROR < RUNTIME | the server failed: " + S->failure + " >");
    if (n > S->pools[integrator].cap || n * (S->dim + 1) > S->pin_res_cap)
        return SUSER("The request is larger than the server's HBM budget allows.");
    r->id = S->next_id++;
    r->t_submit = S->now();
    *id = r->id;
    S->pending.push_back(r->id);
    S->reqs[r->id] = std::move(r);
    ++S->st.submitted;
    S->cv.notify_all();
    return GR_OK;
}

int gr_server_wait(gr_server *S, int64_t id, double timeout_s, int32_t *state) {
    if (!S) return SUSER("null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return SUSER("unknown request");
    Req *r = it->second.get();
    auto finished = [&] { return r->state == GR_REQ_DONE || r->state == GR_REQ_CANCELLED || r->state == GR_REQ_FAILED; };
    if (timeout_s < 0) S->done_cv.wait(lk, finished);
    else S->done_cv.wait_for(lk, std::chrono::duration<double>(timeout_s), finished);
    if (state) *state = r->state;
    if (r->state == GR_REQ_FAILED)
        return sfail(GR_ERR_RUNTIME, "ERROR < RUNTIME | the server failed: " + S->failure + " >");
    return GR_OK;
}

int gr_server_result(gr_server *S, int64_t id, gr_request_info *info, float *positions, int32_t *status,
                     int64_t capacity) {
    if (!S) return SUSER("null server");
    std::lock_guard<std::mutex> g(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return SUSER("unknown request");
    Req *r = it->second.get();
    if (info) {
        info->n = r->n;
        info->dim = S->dim;
        info->integrator = r->integrator;
        info->start_step = r->start_step;
        info->steps = r->end_step - r->start_step;
        info->submit_s = r->t_submit;
        info->admit_s = r->t_admit;
        info->done_s = r->t_done;
        info->state = r->state;
    }
    if (positions || status) {
        if (r->state != GR_REQ_DONE) return SUSER("The request has not completed.");
        if (capacity < r->n) return SUSER("Output buffer too small.");
        if (positions) std::memcpy(positions, r->pos.data(), r->pos.size() * sizeof(float));
        if (status) std::memcpy(status, r->status.data(), r->status.size() * sizeof(int32_t));
    }
    return GR_OK;
}

int gr_server_release(gr_server *S, int64_t id) {
    if (!S) return SUSER("null server");
    std::lock_guard<std::mutex> g(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return SUSER("unknown request");
    Req *r = it->second.get();
    if (r->state == GR_REQ_PENDING || r->state == GR_REQ_ACTIVE)
        return SUSER("The request is still running; cancel it first.");
    if (r->done_ev) cudaEventDestroy(r->done_ev);
    S->reqs.erase(it);
    return GR_OK;
}

int gr_server_cancel(gr_server *S, int64_t id) {
    if (!S) return SUSER("null server");
    std::lock_guard<std::mutex> g(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return SUSER("unknown request");
    Req *r = it->second.get();
    if (r->state == GR_REQ_PENDING) {
        for (auto p = S->pending.begin(); p != S->pending.end(); ++p)
            if (*p == id) {
                S->pending.erase(p);
                break;
            }
        r->state = GR_REQ_CANCELLED;
        std::vector<float>().swap(r->seeds);
        ++S->st.cancelled;
        S->done_cv.notify_all();
    } else if (r->state == GR_REQ_ACTIVE) {
        r->cancelled = true;   // its particles finish with the window it ends in; results dropped
        ++S->st.cancelled;
    }
    return GR_OK;
}

int gr_server_stats_get(gr_server *S, gr_server_stats *out) {
    if (!S || !out) return SUSER("null argument");
    unsigned long long ps = 0;
    SK(cudaSetDevice(S->s.device));
    SK(cudaMemcpy(&ps, S->counters.p, sizeof ps, cudaMemcpyDeviceToHost));
    std::lock_guard<std::mutex> g(S->mu);
    *out = S->st;
    out->particle_steps = (int64_t)ps;
    out->pending = (int64_t)S->pending.size();
    out->active = (int64_t)S->active.size();
    out->clock_steps = (int64_t)S->sched.steps.size();
    out->windows_per_sweep = S->W;
    return GR_OK;
}

void gr_server_destroy(gr_server *S) { delete S; }

}  // extern "C"
