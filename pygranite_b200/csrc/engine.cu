// engine.cu — host engine and C ABI of libgranite_b200.so (declarations: include/granite_b200.h).
//
// Replaces the reference's TrajectoryIntegrator host driver (source/granite/
// TrajectoryIntegrator.tpp:467-1049, TrajectoryIntegrator.cpp:146-693):
//  * snapshot store: a device ring of `ring_slots` snapshots per quantity (reference: a
//    3-slot ring of cudaArray textures filled by synchronous cudaMemcpy3D).  Host data is
//    copied into pinned staging, moved by cudaMemcpyAsync on a copy stream and packed
//    node-major by a kernel; events order the copies against the step launches, so the
//    loader callback and the uploads for the next window overlap the current window.
//  * step loop: one launch advances all particles through one or more windows (the
//    reference launches once per step, synchronises, and copies every saved step to the
//    host); records go to a device history in the (particle, record, component) layout the
//    Python accessors return.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "../../include/granite_b200.h"
#include "expr.h"
#include "host_util.h"
#include "pack_kernels.cuh"
#include "advance.h"
#include "compact.cuh"
#include "engine_graph.h"
#include "granite_kernels.cuh"
#include "jit.h"
#include "schedule.h"

using namespace granite_b200;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define USER_ERR(...) fail(GR_ERR_USER, "ERROR < USER INPUT | " __VA_ARGS__)

}  // namespace

namespace granite_b200 {
// lets other translation units of the library report through gr_last_error()
void set_last_error(const char *msg) { g_last_error = msg ? msg : ""; }
}  // namespace granite_b200

namespace {

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t err_ = (call);                                                                 \
        if (err_ != cudaSuccess)                                                                   \
            return fail(GR_ERR_RUNTIME, "ERROR < RUNTIME | CUDA error | %s : %s, line %d >",       \
                        cudaGetErrorString(err_), __FILE__, __LINE__);                             \
    } while (0)

// ------------------------------------------------------------------ aux kernels

// Seeds (AoS, n x dim) -> state SoA; zeroes the per-particle accumulators.
__global__ void seed_kernel(const float *__restrict__ seeds, int64_t n, int dim, float *px, float *py,
                            float *pz, int32_t *status, int32_t *id, const int32_t *__restrict__ life_src,
                            int32_t *life) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        px[i] = seeds[i * dim];
        py[i] = seeds[i * dim + 1];
        if (dim == 3) pz[i] = seeds[i * dim + 2];
        status[i] = 0;
        id[i] = (int32_t)i;
        if (life_src) life[i] = life_src[i];
    }
}

// Record 0 of the history = the seeds (TrajectoryIntegrator.cpp:424-442): the first row of the
// record-major history.
__global__ void seed_record_kernel(const float *__restrict__ seeds, int64_t n, int dim, float *hpos) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * dim; i += (int64_t)gridDim.x * blockDim.x)
        hpos[i] = seeds[i];
}

// Records of particles that left the live set (retired at compaction) are not written after
// their retirement: they repeat the particle's frozen state, which is substituted when the rows
// are read.  ret[pid] = the first position record not written for pid (a large value for
// particles never retired), frz[pid * D + d] = its frozen value; history row x of the quantity
// belongs to position record rec_of_row ? rec_of_row[x] : x + rec_offset.
struct RowFill {
    const int32_t *ret;
    const float *frz;
    int32_t rec_offset;
    const int32_t *rec_of_row;
};

// Record-major history rows -> particle-major rows: records [r0, r1) of particles [p0, p1), D
// floats each, from src[(r * n + p) * D + d] to dst[((p - p0) * nr + r - r0) * D + d], rows of nr
// records (the layout of TrajectorySet's accessors, TrajectorySet.cpp:110-160), with the frozen
// values of retired particles substituted (RowFill).  A 32-record x 32-particle tile through
// shared memory: reads run along a record row, writes along a particle's records, both coalesced.
template <int D>
__global__ void __launch_bounds__(256) records_to_rows_kernel(const float *__restrict__ src, int64_t n, int32_t r0,
                                                              int32_t r1, int64_t p0, int64_t p1,
                                                              float *__restrict__ dst, int32_t nr, RowFill fill) {
    __shared__ float tile[32][32 * D + 1];
    __shared__ int32_t ret[32];
    const int32_t rt = r0 + (int32_t)blockIdx.y * 32;
    const int64_t pt = p0 + (int64_t)blockIdx.x * 32;
    if (threadIdx.x < 32) ret[threadIdx.x] = (fill.ret && pt + threadIdx.x < p1) ? fill.ret[pt + threadIdx.x] : 0x7fffffff;
    __syncthreads();
    for (int idx = threadIdx.x; idx < 32 * 32 * D; idx += blockDim.x) {
        const int rr = idx / (32 * D), f = idx - rr * (32 * D);
        const int q = f / D;
        if (rt + rr < r1 && pt + q < p1) {
            const int32_t r = rt + rr;
            const int32_t rec = fill.rec_of_row ? fill.rec_of_row[r] : r + fill.rec_offset;
            tile[rr][f] = rec >= ret[q] ? fill.frz[(pt + q) * D + (f - q * D)] : src[((int64_t)r * n + pt) * D + f];
        }
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < 32 * 32 * D; idx += blockDim.x) {
        const int q = idx / (32 * D), g = idx - q * (32 * D);
        const int rr = g / D, d = g - rr * D;
        if (rt + rr < r1 && pt + q < p1)
            dst[((pt + q - p0) * nr + (rt + rr - r0)) * D + d] = tile[rr][q * D + d];
    }
}

// Per-particle retirement of the retired store so far: the first position record the particle
// did not write (its retirement record) and its frozen position, volume / expression values and
// per-step curvature, for RowFill.  Idempotent: runs before each read of the history.
__global__ void note_retired_kernel(StateView R, const int32_t *n_ret, int dim, int nvol, int nexpr, int curv,
                                    int64_t n, int32_t *ret, float *frz_pos, float *frz_vol, float *frz_cmp,
                                    float *frz_curv) {
    const int64_t nr = *n_ret;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nr; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = R.id[j];
        ret[pid] = R.retire[j];
        frz_pos[pid * dim] = R.px[j];
        frz_pos[pid * dim + 1] = R.py[j];
        if (dim == 3) frz_pos[pid * dim + 2] = R.pz[j];
        for (int k = 0; k < nvol; ++k) frz_vol[k * n + pid] = R.volc[k * R.stride + j];
        for (int k = 0; k < nexpr; ++k) frz_cmp[k * n + pid] = R.cmpc[k * R.stride + j];
        if (curv) frz_curv[pid] = R.curv[j];
    }
}

// Writes one record from the state (the SaveInterval == 0 final record, tpp:914-915).
template <int DIM>
__global__ void save_state_kernel(const __grid_constant__ KParams P, int32_t rec, int32_t crec, int32_t irec,
                                  int write_curv) {
    const int64_t n = P.n_dev ? (int64_t)*P.n_dev : P.n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = P.id[i];
        float *hp = P.hpos + ((int64_t)rec * P.n_total + pid) * DIM;
        hp[0] = P.px[i];
        hp[1] = P.py[i];
        if (DIM == 3) hp[2] = P.pz[i];
        if (P.curvature_mode == 3 && write_curv) P.hcurv[(int64_t)crec * P.n_total + pid] = P.curv[i];
        if (P.volume_mode != 0)
            for (int k = 0; k < P.nvol; ++k) P.hvol[((int64_t)k * P.Li + irec) * P.n_total + pid] = P.volc[k * P.n_state + i];
        for (int e = 0; e < P.nexpr; ++e) P.hcmp[((int64_t)e * P.Li + irec) * P.n_total + pid] = P.cmpc[e * P.n_state + i];
    }
}

// State (slot order) -> final per-particle outputs (particle order).
__global__ void finalize_kernel(const __grid_constant__ KParams P, int32_t *status_out, float *length_out,
                                float *tc_out) {
    const int64_t n = P.n_dev ? (int64_t)*P.n_dev : P.n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = P.id[i];
        status_out[pid] = P.status[i];
        if (P.abort_mode != 0) length_out[pid] = P.length[i];
        if (P.curvature_mode != 0) tc_out[pid] = P.tc[i];
    }
}

}  // namespace

struct RunPlan;

struct gr_engine {
    gr_settings s{};
    int dim = 3;
    bool dyn_any = false, wind_dynamic = false;
    cudaStream_t cs = nullptr, xs = nullptr;
    int K = 3;

    // geometry
    bool grid_set = false;
    int64_t nx = 0, ny = 0, nz = 1, nodes = 0;
    float scale[3]{}, off[3]{}, dom[3]{}, inv_scale[3]{};

    // rings
    DevBuf<char> wind;
    int64_t wind_stride = 0;
    bool use_pair = false;             // window-pair layout for the step kernel
    DevBuf<char> pairbuf[2];
    int64_t pair_window[2] = {-1, -1};
    // the next window's pair is packed on ps while the current window's launches run
    cudaStream_t ps = nullptr;
    cudaEvent_t pair_ready[2] = {nullptr, nullptr}, pair_go = nullptr;
    bool pair_pending[2] = {false, false};
    DevBuf<float> vol, cons, lift, topo;
    int nvol = 0, ncon = 0;
    bool has_topo = false, has_uplift = false;
    std::vector<int64_t> wind_holds, vol_holds, cons_holds, lift_holds;
    std::vector<cudaEvent_t> slot_free, slot_ready;
    std::vector<bool> slot_used;
    // device staging of a snapshot's planes, double-buffered: the upload of snapshot s + 1 (on
    // the upload stream us) overlaps the pack of snapshot s, which waits for its ring slot
    DevBuf<float> raw[2];
    int raw_next = 0;
    cudaEvent_t raw_free[2] = {nullptr, nullptr};   // the pack that read raw[j] is done
    cudaStream_t us = nullptr;
    PinnedBuf pin[2];
    int pin_next = 0;
    cudaEvent_t upload_done = nullptr; // end of a DMA straight from a caller's page-locked buffer
    PinnedBuf bounce[2];               // pinned staging of result copies

    // expressions
    Program progs[GR_MAX_EXPR]{};
    int nexpr = 0;
    DevBuf<Program> d_prog;

    // particles
    int64_t n = 0;
    DevBuf<float> seeds;               // AoS n x dim
    struct State {
        DevBuf<float> px, py, pz, qx, qy, qz, kx, ky, kz, lx, ly, lz, length, tc, curv, volc, cmpc;
        DevBuf<float4> vlast;          // inputs of deferred volume / expression values
        DevBuf<int32_t> status, id, retire, life;
    };
    State st[2];                       // double-buffered live state (compaction swaps)
    State ret;                         // retired particles (frozen state)
    State ck;                          // MinimumAliveParticles: state before the current launch
    DevBuf<float4> vrec;               // inputs of a record's deferred volume / expression values
    cudaKernel_t jit_extras = nullptr; // run-time compiled deferred kernel of the expressions (jit.cu)
    std::string jit_why;               // why there is none
    DevBuf<unsigned> alive_at;         // per-step alive counts of a launch, 32 shards per step
    std::vector<unsigned> h_alive;
    int cur = 0;
    bool compacting = false;
    DevBuf<int32_t> d_counts;          // [0] live, [1] live after a pass, [2] retired
    int32_t *h_live = nullptr;         // pinned copy of the live count
    cudaEvent_t live_ready = nullptr;
    DevBuf<int32_t> c_key, c_hist, c_bintab, c_chunk, c_perm;
    int bx = 4, by = 4, bz = 2, nbx = 0, nby = 0, nbz = 0, nbins = 0;

    DevBuf<float> hpos, hcurv, hvol, hcmp;   // record-major (KParams)
    DevBuf<float> stage, sstage;             // particle-major chunks for the fetch / the streaming
    DevBuf<int32_t> ret_rec;                 // retirement record per particle (RowFill)
    DevBuf<float> frz_pos, frz_vol, frz_cmp, frz_curv;   // frozen values of retired particles
    DevBuf<int32_t> rec_of_crec;             // position record of each curvature record
    DevBuf<int32_t> out_status;
    DevBuf<float> out_length, out_tc;
    DevBuf<unsigned long long> counters;
    unsigned long long *h_counters = nullptr;   // pinned
    DevBuf<StepEntry> d_sched;
    std::vector<StepEntry> h_sched;
    int64_t L = 0, Lc = 0, Li = 0;
    std::shared_ptr<RunPlan> plan;     // host plan of the current / last run
    int64_t step_cap = 0;              // > 0: runs stop after this many steps (trial runs)

    // per-particle lifetimes (steps); a particle stops once it has run its lifetime
    DevBuf<int32_t> life_src;
    int64_t life_n = 0;
    int32_t life_max = 0;
    bool has_life = false;

    // graph runs
    uint64_t gen = 0;                  // bumped by every call that may move device buffers
    int64_t graph_executed = 0, graph_records = 0;

    // result streaming (gr_set_result_destinations)
    gr_result_destinations dest{};
    bool dest_set = false;
    bool dest_run = false;             // this run copies into the destinations
    bool dest_during = false;          // ... already while it runs
    int32_t streamed = 0;              // records [0, streamed) are copied or on their way
    cudaStream_t ds = nullptr;         // stream of those copies
    cudaEvent_t ds_ev = nullptr;

    // results
    bool have_result = false;
    gr_result_info info{};
    gr_stats stats{};
    std::vector<cudaEvent_t> ev_pool;

    ~gr_engine() {
        if (cs) cudaStreamSynchronize(cs);
        if (xs) cudaStreamSynchronize(xs);
        if (us) cudaStreamSynchronize(us);
        if (ps) cudaStreamSynchronize(ps);
        for (auto ev : pair_ready)
            if (ev) cudaEventDestroy(ev);
        if (pair_go) cudaEventDestroy(pair_go);
        for (auto e : raw_free)
            if (e) cudaEventDestroy(e);
        for (auto e : slot_free) cudaEventDestroy(e);
        for (auto e : slot_ready) cudaEventDestroy(e);
        for (auto e : ev_pool) cudaEventDestroy(e);
        if (h_counters) gr_host_free(h_counters);
        if (h_live) gr_host_free(h_live);
        if (live_ready) cudaEventDestroy(live_ready);
        if (upload_done) cudaEventDestroy(upload_done);
        if (ds) cudaStreamSynchronize(ds);
        if (ds_ev) cudaEventDestroy(ds_ev);
        if (ds) cudaStreamDestroy(ds);
        if (cs) cudaStreamDestroy(cs);
        if (xs) cudaStreamDestroy(xs);
        if (us) cudaStreamDestroy(us);
        if (ps) cudaStreamDestroy(ps);
    }
};

namespace {

int set_device(gr_engine *e) {
    CK(cudaSetDevice(e->s.device));
    return GR_OK;
}

int ensure_pinned(gr_engine *e, size_t bytes, PinnedBuf *&out) {
    PinnedBuf &b = e->pin[e->pin_next];
    e->pin_next ^= 1;
    if (b.done) CK(cudaEventSynchronize(b.done));
    if (b.bytes < bytes) {
        if (b.p) gr_host_free(b.p);
        b.p = nullptr;
        if (gr_host_alloc((int64_t)bytes, &b.p) != GR_OK) return GR_ERR_RUNTIME;
        b.bytes = bytes;
    }
    if (!b.done) CK(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    out = &b;
    return GR_OK;
}

// True when [p, p + bytes) lies in page-locked host memory known to CUDA (cudaHostAlloc,
// cudaHostRegister, gr_host_alloc): the DMA engines read and write it directly.
bool pinned_range(const void *p, size_t bytes) {
    return bytes > 0 && gr_host_is_pinned(p) && gr_host_is_pinned(static_cast<const char *>(p) + bytes - 1);
}

// Host -> device copy on the copy stream, after whatever the stream already holds.  A
// page-locked source is read by the DMA engine directly, and the call returns once that copy
// is done (the caller may release the source); any other source is staged through the
// double-buffered pinned staging by a parallel host copy.
int upload(gr_engine *e, void *dst, const void *src, size_t bytes) {
    if (pinned_range(src, bytes)) {
        CK(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, e->xs));
        CK(cudaEventRecord(e->upload_done, e->xs));
        CK(cudaEventSynchronize(e->upload_done));
    } else {
        PinnedBuf *pb = nullptr;
        int rc = ensure_pinned(e, bytes, pb);
        if (rc) return rc;
        parallel_memcpy(pb->p, src, bytes);
        CK(cudaMemcpyAsync(dst, pb->p, bytes, cudaMemcpyHostToDevice, e->xs));
        CK(cudaEventRecord(pb->done, e->xs));
    }
    e->stats.h2d_bytes += (int64_t)bytes;
    return GR_OK;
}

int setup_grid(gr_engine *e, int64_t nz, int64_t ny, int64_t nx) {
    if (nx < 1 || ny < 1 || nz < 1) return USER_ERR("Invalid dataset was provided. Empty grid. >");
    if (nx > (1 << 30) || ny > (1 << 30) || nz > (1 << 30) || nx * ny * nz > (int64_t(1) << 40))
        return USER_ERR("Invalid dataset was provided. Grid too large. >");
    e->nx = nx; e->ny = ny; e->nz = e->dim == 3 ? nz : 1;
    e->nodes = e->nx * e->ny * e->nz;
    // the step kernel indexes nodes (and the padded 3D window pair) with 32-bit integers
    if (padded_pair_nodes(e->dim, e->nx, e->ny, e->nz) > (int64_t(1) << 31) - 1)
        return USER_ERR("Invalid dataset was provided. Grid too large. >");
    const gr_settings &s = e->s;
    // GridScale / Offset / Domain (TrajectoryIntegrator.tpp:521-574)
    const float *gs = s.grid_scale, *of = s.offset;
    if (s.grid_scale_len == 1) { e->scale[0] = e->scale[1] = e->scale[2] = gs[0]; }
    else if (s.grid_scale_len == 2) { e->scale[0] = gs[0]; e->scale[1] = gs[1]; e->scale[2] = gs[0]; }
    else if (s.grid_scale_len == 3) { e->scale[0] = gs[0]; e->scale[1] = gs[1]; e->scale[2] = gs[2]; }
    else return USER_ERR("Invalid GridScale dimension. >");
    if (s.offset_len == 1) { e->off[0] = e->off[1] = e->off[2] = of[0]; }
    else if (s.grid_scale_len == 2 && s.offset_len >= 2) { e->off[0] = of[0]; e->off[1] = of[1]; e->off[2] = of[0]; }
    else if (s.grid_scale_len == 3 && s.offset_len >= 3) { e->off[0] = of[0]; e->off[1] = of[1]; e->off[2] = of[2]; }
    else return USER_ERR("Invalid Offset dimension. >");
    const float g[3] = {(float)e->nx, (float)e->ny, (float)(e->dim == 3 ? nz : 0)};
    for (int d = 0; d < 3; ++d) {
        e->dom[d] = g[d] * e->scale[d];
        e->inv_scale[d] = 1.0f / e->scale[d];
    }
    const int bytes_node = e->s.storage == GR_STORE_F32 ? (e->dim == 3 ? 16 : 8) : (e->dim == 3 ? 8 : 4);
    e->wind_stride = ((e->nodes * bytes_node + 255) / 256) * 256;
    CK(e->wind.alloc((size_t)e->wind_stride * e->K));
    for (auto &b : e->raw) CK(b.alloc((size_t)e->nodes * e->dim));
    e->grid_set = true;
    return GR_OK;
}

int wait_slot_free(gr_engine *e, int slot) {
    if (e->slot_used[slot]) CK(cudaStreamWaitEvent(e->xs, e->slot_free[slot], 0));
    return GR_OK;
}

int pack_launch(gr_engine *e, const float *u, const float *v, const float *w, int slot) {
    void *dst = e->wind.p + (int64_t)slot * e->wind_stride;
    const int threads = 256;
    const int blocks = grid_for(e->nodes, threads);
    switch (e->s.storage) {
        case GR_STORE_BF16: pack_wind_kernel<__nv_bfloat16><<<blocks, threads, 0, e->xs>>>(u, v, w, dst, e->nodes, e->dim); break;
        case GR_STORE_F16: pack_wind_kernel<__half><<<blocks, threads, 0, e->xs>>>(u, v, w, dst, e->nodes, e->dim); break;
        default: pack_wind_kernel<float><<<blocks, threads, 0, e->xs>>>(u, v, w, dst, e->nodes, e->dim); break;
    }
    CK(cudaGetLastError());
    e->stats.aux_launches++;
    return GR_OK;
}

int check_shape(gr_engine *e, int64_t nz, int64_t ny, int64_t nx) {
    if (e->dim == 3) {
        if (nz != e->nz) return USER_ERR("Invalid dataset was provided. Shape does not match in z dimension (3D). >");
        if (ny != e->ny) return USER_ERR("Invalid dataset was provided. Shape does not match in y dimension (3D). >");
        if (nx != e->nx) return USER_ERR("Invalid dataset was provided. Shape does not match in x dimension (3D). >");
    } else {
        if (ny != e->ny) return USER_ERR("Invalid dataset was provided. Shape does not match in y dimension (2D). >");
        if (nx != e->nx) return USER_ERR("Invalid dataset was provided. Shape does not match in x dimension (2D). >");
    }
    return GR_OK;
}

int load_wind(gr_engine *e, int64_t snapshot, const float *const *comps, int32_t ncomp, int64_t nz, int64_t ny,
              int64_t nx, bool device_src) {
    if (e) ++e->gen;   // device buffers may move: a captured batch is rebuilt
    if (!e) return USER_ERR("null engine >");
    if (snapshot < 0) return USER_ERR("negative snapshot index >");
    if (ncomp != e->dim)
        return fail(GR_ERR_USER, "%s", e->dim == 3
                        ? "ERROR < USER INPUT | Invalid dataset was provided. Wrong amout of data (3D). >"
                        : "ERROR < USER INPUT | Invalid dataset was provided. Wrong amout of data (2D). >");
    for (int c = 0; c < ncomp; ++c)
        if (!comps || !comps[c]) return USER_ERR("null windfield component >");
    if (e->dim == 2) nz = 1;
    int rc = set_device(e);
    if (rc) return rc;
    if (!e->grid_set) {
        rc = setup_grid(e, nz, ny, nx);
        if (rc) return rc;
    } else {
        rc = check_shape(e, nz, ny, nx);
        if (rc) return rc;
    }
    const int slot = (int)(snapshot % e->K);
    const size_t plane = (size_t)e->nodes;
    // Host planes go to a device staging buffer on the upload stream, which waits only for the
    // pack that last read that buffer (two loads back); the pack into the ring slot, on the
    // copy stream, waits for the upload and for the slot to be released.
    const int j = e->raw_next;
    float *raw[3] = {e->raw[j].p, e->raw[j].p + plane, e->raw[j].p + 2 * plane};
    bool pinned = !device_src;
    for (int c = 0; c < ncomp && pinned; ++c) pinned = pinned_range(comps[c], plane * sizeof(float));
    if (device_src) {
        for (int c = 0; c < ncomp; ++c) raw[c] = const_cast<float *>(comps[c]);
    } else {
        e->raw_next ^= 1;
        CK(cudaStreamWaitEvent(e->us, e->raw_free[j], 0));
        if (pinned) {
            for (int c = 0; c < ncomp; ++c)
                CK(cudaMemcpyAsync(raw[c], comps[c], plane * sizeof(float), cudaMemcpyHostToDevice, e->us));
        } else {
            PinnedBuf *pb = nullptr;
            rc = ensure_pinned(e, plane * ncomp * sizeof(float), pb);
            if (rc) return rc;
            for (int c = 0; c < ncomp; ++c)
                parallel_memcpy(static_cast<float *>(pb->p) + c * plane, comps[c], plane * sizeof(float));
            CK(cudaMemcpyAsync(raw[0], pb->p, plane * ncomp * sizeof(float), cudaMemcpyHostToDevice, e->us));
            CK(cudaEventRecord(pb->done, e->us));
        }
        CK(cudaEventRecord(e->upload_done, e->us));
        CK(cudaStreamWaitEvent(e->xs, e->upload_done, 0));
        e->stats.h2d_bytes += (int64_t)(plane * ncomp * sizeof(float));
    }
    rc = wait_slot_free(e, slot);
    if (rc) return rc;
    rc = pack_launch(e, raw[0], raw[1], e->dim == 3 ? raw[2] : raw[1], slot);
    if (rc) return rc;
    if (!device_src) CK(cudaEventRecord(e->raw_free[j], e->xs));
    CK(cudaEventRecord(e->slot_ready[slot], e->xs));
    if (device_src) CK(cudaStreamSynchronize(e->xs));
    if (pinned) CK(cudaEventSynchronize(e->upload_done));   // the caller may release its planes
    e->wind_holds[slot] = snapshot;
    return GR_OK;
}

int ensure_particles(gr_engine *e) {
    if (e->n <= 0) return USER_ERR("Provided TrajectorySet does not contain any data. >");
    return GR_OK;
}

}  // namespace

// ====================================================================== C ABI

extern "C" {

// Automatic compaction (sort_interval < 0): a Morton re-sort every 8 launches measured best on
// the 3D benchmark configuration (1e6 particles: 2.05e10 against 1.99e10 every 4 and 2.03e10
// every 12); below 65,536 particles the passes cost more than the sorted warps save (the 2D
// double gyre, 10,000 particles: 1.74e10 with them, 1.95e10 without).
constexpr int kAutoSortInterval = 8;
constexpr int64_t kAutoSortMin = 65536;

void gr_settings_default(gr_settings *s) {
    std::memset(s, 0, sizeof *s);
    s->space = 0;
    s->integrator = 1;
    s->windfield_mode = 1;
    s->delta_t = 1.f;
    s->data_time_distance = 60.f;
    s->grid_scale[0] = s->grid_scale[1] = s->grid_scale[2] = 25.f;
    s->grid_scale_len = 3;
    s->offset_len = 3;
    s->save_interval = 1;
    s->maximum_simulation_time = 100.f;
    s->sort_interval = -1;  // automatic: kAutoSortInterval launches from kAutoSortMin particles, else off
}

const char *gr_last_error(void) { return g_last_error.c_str(); }

int gr_create(const gr_settings *settings, gr_engine **out) {
    g_last_error.clear();
    if (!settings || !out) return USER_ERR("null argument >");
    *out = nullptr;
    const gr_settings &s = *settings;
    if (s.space != 0 && s.space != 1) return USER_ERR("Invalid Space. >");
    if (s.delta_t <= 0.f || !std::isfinite(s.delta_t)) return USER_ERR("DeltaT must be positive. >");
    if (s.data_time_distance <= 0.f || !std::isfinite(s.data_time_distance))
        return USER_ERR("DataTimeDistance must be positive. >");
    if (!std::isfinite(s.maximum_simulation_time)) return USER_ERR("MaximumSimulationTime must be finite. >");
    if (s.maximum_simulation_time / s.delta_t > 5.0e8f) return USER_ERR("Too many integration steps requested. >");
    if (s.save_interval < 0) return USER_ERR("SaveInterval must not be negative. >");
    if (s.storage < 0 || s.storage > 2) return USER_ERR("Invalid storage type. >");
    if (s.filter_weights < 0 || s.filter_weights > 1) return USER_ERR("Invalid filter weights. >");
    auto e = std::make_unique<gr_engine>();
    e->s = s;
    e->dim = s.space == 0 ? 3 : 2;
    if (e->dim == 2) e->s.uplift_mode = 0;   // 2D variants force uplift Off (TrajectoryIntegratorMacros.hpp:67)
    e->wind_dynamic = s.windfield_mode == 1;
    e->dyn_any = e->wind_dynamic || e->s.uplift_mode == 2 || s.volume_mode == 2 || s.constants_mode == 2;
    e->K = s.ring_slots >= 3 ? s.ring_slots : 3;
    if (e->K > 100000) return USER_ERR("ring_slots too large >");
    CK(cudaSetDevice(s.device));
    CK(cudaStreamCreateWithFlags(&e->cs, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->xs, cudaStreamNonBlocking));
    e->slot_free.resize(e->K);
    e->slot_ready.resize(e->K);
    e->slot_used.assign(e->K, false);
    for (int k = 0; k < e->K; ++k) {
        CK(cudaEventCreateWithFlags(&e->slot_free[k], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&e->slot_ready[k], cudaEventDisableTiming));
    }
    CK(cudaEventCreateWithFlags(&e->upload_done, cudaEventDisableTiming));
    CK(cudaStreamCreateWithFlags(&e->us, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&e->ps, cudaStreamNonBlocking));
    for (auto &ev : e->pair_ready) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    CK(cudaEventCreateWithFlags(&e->pair_go, cudaEventDisableTiming));
    for (auto &ev : e->raw_free) CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    e->wind_holds.assign(e->K, -1);
    e->vol_holds.assign(e->K, -1);
    e->cons_holds.assign(e->K, -1);
    e->lift_holds.assign(e->K, -1);
    CK(e->counters.alloc(4));
    // small page-locked words from the host cache: no page-locking per engine
    if (gr_host_alloc(4 * sizeof(unsigned long long), reinterpret_cast<void **>(&e->h_counters)) != GR_OK)
        return GR_ERR_RUNTIME;
    *out = e.release();
    return GR_OK;
}

void gr_destroy(gr_engine *engine) { delete engine; }

int gr_load_windfield(gr_engine *e, int64_t snapshot, const float *const *comps, int32_t ncomp, int64_t nz,
                      int64_t ny, int64_t nx) {
    return load_wind(e, snapshot, comps, ncomp, nz, ny, nx, false);
}

int gr_load_windfield_device(gr_engine *e, int64_t snapshot, const float *const *comps, int32_t ncomp, int64_t nz,
                             int64_t ny, int64_t nx) {
    return load_wind(e, snapshot, comps, ncomp, nz, ny, nx, true);
}

int gr_load_volume(gr_engine *e, int64_t snapshot, int32_t index, const float *data, int64_t nz, int64_t ny,
                   int64_t nx) {
    if (e) ++e->gen;   // device buffers may move: a captured batch is rebuilt
    if (!e || !data) return USER_ERR("null argument >");
    if (index < 0 || index >= GR_MAX_VOLUMES) return USER_ERR("You provided more additional volumes than supported. >");
    if (!e->grid_set) return USER_ERR("The windfield must be loaded before additional volumes. >");
    if (e->dim == 2) nz = 1;
    int rc = check_shape(e, nz, ny, nx);
    if (rc) return rc;
    rc = set_device(e);
    if (rc) return rc;
    CK(e->vol.alloc((size_t)e->nodes * GR_MAX_VOLUMES * e->K));
    const int slot = (int)(snapshot % e->K);
    rc = wait_slot_free(e, slot);
    if (rc) return rc;
    float *dst = e->vol.p + ((int64_t)slot * GR_MAX_VOLUMES + index) * e->nodes;
    rc = upload(e, dst, data, (size_t)e->nodes * sizeof(float));
    if (rc) return rc;
    CK(cudaEventRecord(e->slot_ready[slot], e->xs));
    if (snapshot == 0 && index + 1 > e->nvol) e->nvol = index + 1;
    e->vol_holds[slot] = snapshot;
    return GR_OK;
}

int gr_load_constant(gr_engine *e, int64_t snapshot, int32_t index, const float *data, int64_t n) {
    if (e) ++e->gen;   // device buffers may move: a captured batch is rebuilt
    if (!e || !data) return USER_ERR("null argument >");
    if (index < 0 || index >= GR_MAX_CONSTANTS) return USER_ERR("You provided more constants than supported. >");
    if (e->n <= 0) return USER_ERR("Seeds must be set before constants. >");
    if (n != e->n) return USER_ERR("Constant dimension does not match number of particles. >");
    int rc = set_device(e);
    if (rc) return rc;
    CK(e->cons.alloc((size_t)e->n * GR_MAX_CONSTANTS * e->K));
    const int slot = (int)(snapshot % e->K);
    rc = wait_slot_free(e, slot);
    if (rc) return rc;
    rc = upload(e, e->cons.p + ((int64_t)slot * GR_MAX_CONSTANTS + index) * e->n, data, (size_t)n * sizeof(float));
    if (rc) return rc;
    CK(cudaEventRecord(e->slot_ready[slot], e->xs));
    if (snapshot == 0 && index + 1 > e->ncon) e->ncon = index + 1;
    e->cons_holds[slot] = snapshot;
    return GR_OK;
}

int gr_load_uplift(gr_engine *e, int64_t snapshot, const float *data, int64_t n, int32_t dim) {
    if (e) ++e->gen;   // device buffers may move: a captured batch is rebuilt
    if (!e || !data) return USER_ERR("null argument >");
    if (e->n <= 0) return USER_ERR("Seeds must be set before the uplift. >");
    if (n != e->n) return USER_ERR("Uplift dimension does not match number of particles. >");
    if (dim != e->dim) return USER_ERR("Uplift dimension does not match the integrator space. >");
    if (e->dim == 2) return GR_OK;   // 2D variants never read the uplift
    int rc = set_device(e);
    if (rc) return rc;
    CK(e->lift.alloc((size_t)e->n * 3 * e->K));
    const int slot = (int)(snapshot % e->K);
    rc = wait_slot_free(e, slot);
    if (rc) return rc;
    rc = upload(e, e->lift.p + (int64_t)slot * e->n * 3, data, (size_t)n * 3 * sizeof(float));
    if (rc) return rc;
    CK(cudaEventRecord(e->slot_ready[slot], e->xs));
    e->has_uplift = true;
    e->lift_holds[slot] = snapshot;
    return GR_OK;
}

int gr_set_topography(gr_engine *e, const float *data, int64_t ny, int64_t nx) {
    if (e) ++e->gen;   // device buffers may move: a captured batch is rebuilt
    if (!e || !data) return USER_ERR("null argument >");
    if (!e->grid_set) return USER_ERR("The windfield must be loaded before the topography. >");
    if (nx != e->nx || ny != e->ny) return USER_ERR("Topography dimensions does not match to provided data! >");
    int rc = set_device(e);
    if (rc) return rc;
    CK(e->topo.alloc((size_t)nx * ny));
    CK(cudaMemcpy(e->topo.p, data, (size_t)nx * ny * sizeof(float), cudaMemcpyHostToDevice));
    e->has_topo = e->dim == 3;   // 2D variants never use the topography (Macros.hpp:71)
    return GR_OK;
}

int gr_compile_expression(gr_engine *e, int32_t index, const char *code, const char *const *volume_names,
                          int32_t n_volumes, const char *const *constant_names, int32_t n_constants) {
    if (e) ++e->gen;   // device buffers may move: a captured batch is rebuilt
    if (!e || !code) return USER_ERR("null argument >");
    if (index < 0 || index >= GR_MAX_EXPRESSIONS) return USER_ERR("At most 4 AdditionalCompute expressions are supported. >");
    std::vector<std::string> vn, cn;
    for (int k = 0; k < n_volumes; ++k) vn.emplace_back(volume_names[k] ? volume_names[k] : "");
    for (int k = 0; k < n_constants; ++k) cn.emplace_back(constant_names[k] ? constant_names[k] : "");
    std::string err;
    Program p{};
    if (!compile_expression(code, vn, cn, e->dim, e->s.curvature_mode, p, err)) return fail(GR_ERR_USER, "%s", err.c_str());
    e->progs[index] = p;
    if (index + 1 > e->nexpr) e->nexpr = index + 1;
    return GR_OK;
}

int gr_plan(const gr_settings *settings, gr_plan_info *out, int64_t capacity, int64_t *window, int32_t *flags,
            float *weights) {
    if (!settings || !out) return USER_ERR("null argument >");
    const gr_settings &s = *settings;
    if (s.delta_t <= 0.f || !std::isfinite(s.delta_t)) return USER_ERR("DeltaT must be positive. >");
    if (s.data_time_distance <= 0.f || !std::isfinite(s.data_time_distance))
        return USER_ERR("DataTimeDistance must be positive. >");
    if (!std::isfinite(s.maximum_simulation_time) || s.maximum_simulation_time / s.delta_t > 5.0e8f)
        return USER_ERR("Too many integration steps requested. >");
    ScheduleInput si;
    const int up = s.space == 0 ? s.uplift_mode : 0;
    si.wind_dynamic = s.windfield_mode == 1;
    si.dyn_any = si.wind_dynamic || up == 2 || s.volume_mode == 2 || s.constants_mode == 2;
    si.delta_t = s.delta_t;
    si.data_time_distance = s.data_time_distance;
    si.maximum_simulation_time = s.maximum_simulation_time;
    si.save_interval = s.save_interval;
    si.time_mode = s.time_mode;
    const Schedule sc = build_schedule(si);
    const int64_t n = (int64_t)sc.steps.size();
    int64_t saves = 0, csaves = 0;
    for (int64_t k = 0; k < n; ++k) {
        const HostStep &h = sc.steps[k];
        saves += h.save;
        csaves += h.save && h.time_pos;
        if (k < capacity) {
            if (window) window[k] = h.window;
            if (flags) flags[k] = (h.save ? 1 : 0) | (h.time_pos ? 2 : 0);
            if (weights) {
                weights[3 * k] = h.t0;
                weights[3 * k + 1] = h.t1;
                weights[3 * k + 2] = h.t2;
            }
        }
    }
    const bool final_rec = s.save_interval == 0;
    out->steps = n;
    out->windows = (int64_t)sc.window_begin.size() - 1;
    out->records = 1 + saves + (final_rec ? 1 : 0);
    out->info_records = saves + (final_rec ? 1 : 0);
    out->curvature_records = s.curvature_mode == 3 ? csaves + ((final_rec && n > 0) ? 1 : 0) : 0;
    return GR_OK;
}

int gr_expression_evaluate(const char *code, const char *const *volume_names, int32_t n_volumes,
                           const char *const *constant_names, int32_t n_constants, int32_t dim,
                           int32_t curvature_mode, const float *ref, float *out) {
    if (!code || !ref || !out) return USER_ERR("null argument >");
    std::vector<std::string> vn, cn;
    for (int k = 0; k < n_volumes; ++k) vn.emplace_back(volume_names[k] ? volume_names[k] : "");
    for (int k = 0; k < n_constants; ++k) cn.emplace_back(constant_names[k] ? constant_names[k] : "");
    std::string err;
    Program p{};
    if (!compile_expression(code, vn, cn, dim, curvature_mode, p, err)) return fail(GR_ERR_USER, "%s", err.c_str());
    *out = evaluate(p, ref);
    return GR_OK;
}

static int set_seeds(gr_engine *e, const float *pos, int64_t n, int32_t dim, bool device_src) {
    if (!e || (!pos && n > 0)) return USER_ERR("null argument >");
    // a captured batch reads the seed buffer when it replays: only a new count or a moved
    // buffer makes it capture again
    const float *before = e->seeds.p;
    const int64_t n_before = e->n;
    struct Bump {
        gr_engine *e;
        const float *p;
        int64_t n;
        ~Bump() { if (e->seeds.p != p || e->n != n) ++e->gen; }
    } bump{e, before, n_before};
    if (dim != e->dim) return USER_ERR("Dimensions of IntegratorSettings and provided TrajectorySet do not match. >");
    if (n <= 0) return USER_ERR("Provided TrajectorySet does not contain any data. >");
    if (n > (int64_t(1) << 31) - 1) return USER_ERR("Too many particles. >");
    int rc = set_device(e);
    if (rc) return rc;
    e->n = n;
    CK(e->seeds.alloc((size_t)n * dim));
    CK(cudaMemcpy(e->seeds.p, pos, (size_t)n * dim * sizeof(float),
                  device_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice));
    if (!device_src) e->stats.h2d_bytes += n * dim * (int64_t)sizeof(float);
    return GR_OK;
}

int gr_set_seeds(gr_engine *e, const float *pos, int64_t n, int32_t dim) { return set_seeds(e, pos, n, dim, false); }
int gr_set_seeds_device(gr_engine *e, const float *pos, int64_t n, int32_t dim) { return set_seeds(e, pos, n, dim, true); }

int gr_set_lifetimes(gr_engine *e, const int32_t *steps, int64_t n) {
    if (!e) return USER_ERR("null engine >");
    ++e->gen;
    if (!steps || n == 0) {
        e->has_life = false;
        e->life_n = 0;
        e->life_max = 0;
        return GR_OK;
    }
    if (n < 0 || n > (int64_t(1) << 31) - 1) return USER_ERR("Invalid lifetime count. >");
    int32_t mx = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (steps[i] < 0) return USER_ERR("Lifetimes must not be negative. >");
        mx = std::max(mx, steps[i]);
    }
    int rc = set_device(e);
    if (rc) return rc;
    CK(e->life_src.alloc((size_t)n));
    CK(cudaMemcpy(e->life_src.p, steps, (size_t)n * sizeof(int32_t), cudaMemcpyHostToDevice));
    e->stats.h2d_bytes += n * (int64_t)sizeof(int32_t);
    e->has_life = true;
    e->life_n = n;
    e->life_max = mx;
    return GR_OK;
}

int gr_update_settings(gr_engine *e, const gr_settings *s) {
    if (!e || !s) return USER_ERR("null argument >");
    const gr_settings &o = e->s;
    // what the loaded data and the ring were built for stays fixed
    const bool same = s->space == o.space && s->windfield_mode == o.windfield_mode &&
                      s->constants_mode == o.constants_mode && s->volume_mode == o.volume_mode &&
                      (e->dim == 2 || s->uplift_mode == o.uplift_mode) && s->storage == o.storage &&
                      (s->ring_slots >= 3 ? s->ring_slots : 3) == e->K && s->device == o.device &&
                      s->grid_scale_len == o.grid_scale_len && s->offset_len == o.offset_len &&
                      std::memcmp(s->grid_scale, o.grid_scale, sizeof o.grid_scale) == 0 &&
                      std::memcmp(s->offset, o.offset, sizeof o.offset) == 0;
    if (!same)
        return USER_ERR("Only run options can change after creation (space, modes, grid, storage, ring and device are fixed). >");
    if (s->delta_t <= 0.f || !std::isfinite(s->delta_t)) return USER_ERR("DeltaT must be positive. >");
    if (s->data_time_distance <= 0.f || !std::isfinite(s->data_time_distance))
        return USER_ERR("DataTimeDistance must be positive. >");
    if (!std::isfinite(s->maximum_simulation_time)) return USER_ERR("MaximumSimulationTime must be finite. >");
    if (s->maximum_simulation_time / s->delta_t > 5.0e8f) return USER_ERR("Too many integration steps requested. >");
    if (s->save_interval < 0) return USER_ERR("SaveInterval must not be negative. >");
    if (s->filter_weights < 0 || s->filter_weights > 1) return USER_ERR("Invalid filter weights. >");
    ++e->gen;
    const int32_t uplift = e->s.uplift_mode;
    e->s = *s;
    e->s.uplift_mode = uplift;
    return GR_OK;
}

int gr_settings_get(const gr_engine *e, gr_settings *out) {
    if (!e || !out) return USER_ERR("null argument >");
    *out = e->s;
    return GR_OK;
}

}  // extern "C"

// ====================================================================== run

// Host plan of one run: the step schedule, record bookkeeping and launch granularity.
struct RunPlan {
    Schedule sched;
    int64_t nsteps = 0, nwin = 0;
    std::vector<int32_t> rec_before;   // records written before step k: 1 + saves in [0, k)
    std::vector<int64_t> save_next;    // first save step >= k (nsteps if none)
    int64_t spl = 0;                   // steps per launch
    bool graph = false;                // fixed launch shapes and no host reads (graph capture)
};

namespace {

int alloc_set(gr_engine *e, gr_engine::State &S, bool retired) {
    const size_t N = (size_t)e->n;
    const int cm = e->s.curvature_mode;
    CK(S.px.alloc(N)); CK(S.py.alloc(N));
    if (e->dim == 3) CK(S.pz.alloc(N));
    CK(S.status.alloc(N)); CK(S.id.alloc(N));
    if (retired) CK(S.retire.alloc(N));
    if (!retired && e->has_life) CK(S.life.alloc(N));
    if (!retired && (cm == 1 || cm == 3)) { CK(S.qx.alloc(N)); CK(S.qy.alloc(N)); CK(S.qz.alloc(N)); }
    if (!retired && e->s.compensated) { CK(S.kx.alloc(N)); CK(S.ky.alloc(N)); CK(S.kz.alloc(N)); }
    if (!retired && cm == 2) { CK(S.lx.alloc(N)); CK(S.ly.alloc(N)); CK(S.lz.alloc(N)); }
    CK(S.length.alloc(N)); CK(S.tc.alloc(N)); CK(S.curv.alloc(N));
    const int nv = std::max(1, e->nvol), ne = std::max(1, e->nexpr);
    CK(S.volc.alloc(N * nv)); CK(S.cmpc.alloc(N * ne));
    const bool extras = (e->s.volume_mode != 0 && e->nvol > 0) || e->nexpr > 0;
    if (!retired && extras) CK(S.vlast.alloc(N));
    return GR_OK;
}

// Device buffers and host tables of a run; enqueues no device work.
int alloc_state(gr_engine *e) {
    const size_t N = (size_t)e->n;
    int rc = alloc_set(e, e->st[0], false);
    if (rc) return rc;
    if (e->st[0].vlast.p) CK(e->vrec.alloc(2 * N));
    CK(e->out_status.alloc(N)); CK(e->out_length.alloc(N)); CK(e->out_tc.alloc(N));
    e->compacting = e->s.sort_interval > 0 || (e->s.sort_interval < 0 && e->n >= kAutoSortMin);
    CK(e->d_counts.alloc(4));
    if (!e->compacting) return GR_OK;
    rc = alloc_set(e, e->st[1], false);
    if (rc) return rc;
    rc = alloc_set(e, e->ret, true);
    if (rc) return rc;
    CK(e->c_key.alloc(N));
    if (!e->h_live && gr_host_alloc(sizeof(int32_t), reinterpret_cast<void **>(&e->h_live)) != GR_OK)
        return GR_ERR_RUNTIME;
    if (!e->live_ready) CK(cudaEventCreateWithFlags(&e->live_ready, cudaEventDisableTiming));
    if (e->nbins == 0) {
        // Morton-ranked brick table (bricks of bx x by x bz nodes)
        e->bx = 4; e->by = 4; e->bz = e->dim == 3 ? 2 : 1;
        for (;;) {
            e->nbx = (int)((e->nx + e->bx - 1) / e->bx);
            e->nby = (int)((e->ny + e->by - 1) / e->by);
            e->nbz = (int)((e->nz + e->bz - 1) / e->bz);
            if ((int64_t)e->nbx * e->nby * e->nbz <= (1 << 20) && e->nbx <= 1024 && e->nby <= 1024 && e->nbz <= 1024) break;
            e->bx *= 2; e->by *= 2; if (e->dim == 3) e->bz *= 2;
        }
        e->nbins = e->nbx * e->nby * e->nbz;
        auto spread = [](uint32_t v) {
            uint64_t x = v & 0x3ff;
            x = (x | (x << 16)) & 0x030000FF;
            x = (x | (x << 8)) & 0x0300F00F;
            x = (x | (x << 4)) & 0x030C30C3;
            x = (x | (x << 2)) & 0x09249249;
            return x;
        };
        std::vector<std::pair<uint64_t, int32_t>> codes((size_t)e->nbins);
        for (int z = 0; z < e->nbz; ++z)
            for (int y = 0; y < e->nby; ++y)
                for (int x = 0; x < e->nbx; ++x) {
                    const int32_t lin = (z * e->nby + y) * e->nbx + x;
                    codes[lin] = {spread(x) | (spread(y) << 1) | (spread(z) << 2), lin};
                }
        std::sort(codes.begin(), codes.end());
        std::vector<int32_t> tab((size_t)e->nbins);
        for (int32_t r = 0; r < e->nbins; ++r) tab[codes[r].second] = r;
        CK(e->c_bintab.alloc(tab.size()));
        CK(cudaMemcpy(e->c_bintab.p, tab.data(), tab.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    }
    CK(e->c_hist.alloc((size_t)e->nbins + 1));
    CK(e->c_chunk.alloc((size_t)(e->nbins + 1 + SCAN_CHUNK - 1) / SCAN_CHUNK));
    CK(e->c_perm.alloc(N));
    return GR_OK;
}

__global__ void init_counts_kernel(int32_t *counts, int32_t n) {
    counts[0] = n;   // live
    counts[1] = n;   // live after the last pass
    counts[2] = 0;   // retired
    counts[3] = 0;
}

// Device start of a run on the compute stream: zeroed accumulators and counters, live and
// retired counts, seeds -> state, record 0.  Capturable.
int reset_state(gr_engine *e) {
    const int64_t n = e->n;
    const size_t N = (size_t)n;
    e->cur = 0;
    gr_engine::State &S = e->st[0];
    if (e->s.compensated) {
        CK(cudaMemsetAsync(S.kx.p, 0, N * 4, e->cs)); CK(cudaMemsetAsync(S.ky.p, 0, N * 4, e->cs));
        CK(cudaMemsetAsync(S.kz.p, 0, N * 4, e->cs));
    }
    if (e->s.curvature_mode == 2) {
        CK(cudaMemsetAsync(S.lx.p, 0, N * 4, e->cs)); CK(cudaMemsetAsync(S.ly.p, 0, N * 4, e->cs));
        CK(cudaMemsetAsync(S.lz.p, 0, N * 4, e->cs));
    }
    CK(cudaMemsetAsync(S.length.p, 0, N * 4, e->cs));
    CK(cudaMemsetAsync(S.tc.p, 0, N * 4, e->cs));
    CK(cudaMemsetAsync(S.curv.p, 0, N * 4, e->cs));
    const int nv = std::max(1, e->nvol), ne = std::max(1, e->nexpr);
    CK(cudaMemsetAsync(S.volc.p, 0, N * nv * 4, e->cs));
    CK(cudaMemsetAsync(S.cmpc.p, 0, N * ne * 4, e->cs));
    if (S.vlast.p) CK(cudaMemsetAsync(S.vlast.p, 0xff, N * sizeof(float4), e->cs));   // step index -1
    init_counts_kernel<<<1, 1, 0, e->cs>>>(e->d_counts.p, (int32_t)n);
    const int threads = 256;
    seed_kernel<<<grid_for(n, threads), threads, 0, e->cs>>>(e->seeds.p, n, e->dim, S.px.p, S.py.p, S.pz.p,
                                                             S.status.p, S.id.p,
                                                             e->has_life ? e->life_src.p : nullptr, S.life.p);
    seed_record_kernel<<<grid_for(n * e->dim, threads), threads, 0, e->cs>>>(e->seeds.p, n, e->dim, e->hpos.p);
    CK(cudaGetLastError());
    if (e->ret_rec.p) CK(cudaMemsetAsync(e->ret_rec.p, 0x7f, (size_t)n * sizeof(int32_t), e->cs));   // never retired
    CK(cudaMemsetAsync(e->counters.p, 0, 4 * sizeof(unsigned long long), e->cs));
    if (e->compacting) *e->h_live = (int32_t)n;
    e->stats.aux_launches += 3;
    return GR_OK;
}

// Snapshots 0 .. m-1 resident in the ring for every quantity the run reloads per snapshot.
int64_t resident_prefix(const gr_engine *e) {
    const bool vol_dyn = e->s.volume_mode == 2 && e->nvol > 0;
    const bool con_dyn = e->s.constants_mode == 2 && e->ncon > 0;
    const bool lift_dyn = e->s.uplift_mode == 2 && e->has_uplift;
    int64_t m = 0;
    for (; m < e->K; ++m) {
        const bool wind_ok = e->wind_dynamic ? e->wind_holds[m] == m : (m > 0 || e->wind_holds[0] == 0);
        if (!wind_ok || (vol_dyn && e->vol_holds[m] != m) || (con_dyn && e->cons_holds[m] != m) ||
            (lift_dyn && e->lift_holds[m] != m))
            break;
    }
    return m;
}

// MinimumAliveParticles: steps per launch are capped so that their alive counts fit alive_at.
constexpr int64_t kAliveSteps = 256;

// Device copy of the particle state a step launch writes (checkpoint / rollback).
int copy_state(gr_engine *e, gr_engine::State &d, gr_engine::State &src, int64_t n) {
    const size_t N = (size_t)e->n, c = (size_t)n;
    auto cp = [&](auto &dst, auto &from, size_t count) -> cudaError_t {
        if (!from.p || !dst.p || count == 0) return cudaSuccess;
        return cudaMemcpyAsync(dst.p, from.p, count * sizeof(*from.p), cudaMemcpyDeviceToDevice, e->cs);
    };
    CK(cp(d.px, src.px, c)); CK(cp(d.py, src.py, c)); CK(cp(d.pz, src.pz, c));
    CK(cp(d.qx, src.qx, c)); CK(cp(d.qy, src.qy, c)); CK(cp(d.qz, src.qz, c));
    CK(cp(d.kx, src.kx, c)); CK(cp(d.ky, src.ky, c)); CK(cp(d.kz, src.kz, c));
    CK(cp(d.lx, src.lx, c)); CK(cp(d.ly, src.ly, c)); CK(cp(d.lz, src.lz, c));
    CK(cp(d.status, src.status, c));
    CK(cp(d.length, src.length, c)); CK(cp(d.tc, src.tc, c)); CK(cp(d.curv, src.curv, c));
    const int nv = std::max(1, e->nvol), ne = std::max(1, e->nexpr);
    for (int k = 0; k < nv; ++k)
        CK(cudaMemcpyAsync(d.volc.p + k * N, src.volc.p + k * N, c * 4, cudaMemcpyDeviceToDevice, e->cs));
    for (int k = 0; k < ne; ++k)
        CK(cudaMemcpyAsync(d.cmpc.p + k * N, src.cmpc.p + k * N, c * 4, cudaMemcpyDeviceToDevice, e->cs));
    return GR_OK;
}

// Keeps the first `steps` steps of a schedule.
void truncate_schedule(Schedule &sc, int64_t steps) {
    if ((int64_t)sc.steps.size() <= steps) return;
    sc.steps.resize((size_t)steps);
    std::vector<int64_t> wb;
    for (int64_t b : sc.window_begin)
        if (b < steps) wb.push_back(b);
    wb.push_back(steps);
    sc.window_begin = wb;
}

// Channel-record index of each position record, for records written in steps [0, executed).
// Position record of each curvature record (curvature records are written at position records
// whose step had data.Time > 0, tpp:997-1012), for RowFill; unused entries hold a large value.
std::vector<int32_t> rec_of_crec_table(const gr_engine *e, const RunPlan &R, int64_t executed) {
    std::vector<int32_t> t((size_t)std::max<int64_t>(1, e->Lc), 0x7fffffff);
    int64_t rr = 1, cc = 0;
    for (int64_t k = 0; k < executed; ++k)
        if (R.sched.steps[k].save) {
            if (R.sched.steps[k].time_pos && cc < (int64_t)t.size()) t[(size_t)cc++] = (int32_t)rr;
            ++rr;
        }
    if (e->s.save_interval == 0 && executed > 0 && cc < (int64_t)t.size()) t[(size_t)cc] = (int32_t)rr;   // the final record
    return t;
}

int ensure_pair(gr_engine *e, int64_t w);
int settle_pairs(gr_engine *e);

int pair_elem(const gr_engine *e) {
    return e->s.storage == GR_STORE_F32 ? (e->dim == 3 ? 16 : 8) : (e->dim == 3 ? 8 : 4);
}

// Bytes of one window-pair buffer: pairs carry a border (pair_pack_padded_kernel,
// pair_pack_edge2_kernel).
size_t pair_bytes(const gr_engine *e) {
    return (size_t)padded_pair_nodes(e->dim, e->nx, e->ny, e->nz) * 2 * pair_elem(e);
}

// Validation, schedule, device schedule and programs, state and history buffers.
int run_prepare(gr_engine *e, RunPlan &R, bool graph) {
    if (!e) return USER_ERR("null engine >");
    g_last_error.clear();
    int rc = set_device(e);
    if (rc) return rc;
    rc = ensure_particles(e);
    if (rc) return rc;
    if (!e->grid_set) return USER_ERR("No windfield was loaded. >");
    if (e->wind_holds[0] != 0)
        return USER_ERR("Snapshot 0 is no longer resident in the ring; load the data again to run again. >");
    if (e->dyn_any && e->wind_dynamic && e->wind_holds[1 % e->K] != 1) return USER_ERR("Cannot increment loader. >");
    const gr_settings &s = e->s;
    // settings combinations the reference has no kernel variant for
    // (TrajectoryIntegrator.gen.py:52-53 and the 2D curvature axis, gen.py:184-187)
    if (e->dim == 2 && (s.curvature_mode == 1 || s.curvature_mode == 3))
        return USER_ERR("No kernel could be picked for your settings configuration. >");
    if (s.constants_mode != 0 && e->nexpr == 0)
        return USER_ERR("No kernel could be picked for your settings configuration. >");
    if (e->has_life && e->life_n != e->n)
        return USER_ERR("Lifetimes were set for %lld particles but the set holds %lld. >", (long long)e->life_n,
                        (long long)e->n);
    if (graph && s.minimum_alive > 0)
        return USER_ERR("MinimumAliveParticles needs host decisions between steps; it cannot run in a graph. >");
    e->have_result = false;
    ++e->gen;
    e->streamed = 0;   // records copied out by result streaming (stream_begin turns it on)
    e->dest_run = e->dest_during = false;
    {
        const int64_t h2d = e->stats.h2d_bytes, d2h = e->stats.d2h_bytes;
        e->stats = gr_stats{};
        e->stats.h2d_bytes = h2d;
        e->stats.d2h_bytes = d2h;
    }

    ScheduleInput si;
    si.dyn_any = e->dyn_any;
    si.wind_dynamic = e->wind_dynamic;
    si.delta_t = s.delta_t;
    si.data_time_distance = s.data_time_distance;
    si.maximum_simulation_time = s.maximum_simulation_time;
    si.save_interval = s.save_interval;
    si.time_mode = s.time_mode;
    R = RunPlan{};
    R.graph = graph;
    R.sched = build_schedule(si);
    // nothing runs after the longest lifetime
    if (e->has_life) truncate_schedule(R.sched, std::max<int64_t>(0, e->life_max));
    if (e->step_cap > 0) truncate_schedule(R.sched, e->step_cap);
    if (graph) {
        // a graph run covers the windows whose snapshots are all resident now
        const int64_t m = resident_prefix(e);
        const int64_t nw = (int64_t)R.sched.window_begin.size() - 1;
        if (e->dyn_any) {
            if (m < 2) return USER_ERR("A graph run needs snapshots 0 and 1 resident in the ring. >");
            if (m - 1 < nw) truncate_schedule(R.sched, R.sched.window_begin[m - 1]);
        }
    }
    R.nsteps = (int64_t)R.sched.steps.size();
    R.nwin = (int64_t)R.sched.window_begin.size() - 1;

    // records: seed + saves (+ the final record when SaveInterval == 0)
    int64_t nsaves = 0;
    for (const auto &st : R.sched.steps) nsaves += st.save;
    e->L = 1 + nsaves + (s.save_interval == 0 ? 1 : 0);
    e->Li = e->L - 1;
    e->Lc = s.curvature_mode == 3 ? e->L - 1 : 0;

    // device schedule
    e->h_sched.resize(std::max<int64_t>(1, R.nsteps));
    {
        int64_t rec = 1, crec = 0, irec = 0;
        for (int64_t k = 0; k < R.nsteps; ++k) {
            const HostStep &h = R.sched.steps[k];
            StepEntry E{};
            E.t0 = h.t0; E.t1 = h.t1; E.t2 = h.t2;
            E.flags = (h.save ? SF_SAVE : 0) | (h.time_pos ? SF_TIME_POS : 0) |
                      (h.save && h.time_pos ? SF_CURV_REC : 0);
            E.rec = (int32_t)rec; E.crec = (int32_t)crec; E.irec = (int32_t)irec;
            E.slot_back = (int32_t)(h.window % e->K);
            E.slot_front = (int32_t)((h.window + 1) % e->K);
            if (h.save) {
                ++rec;
                ++irec;
                if (h.time_pos) ++crec;
            }
            e->h_sched[k] = E;
        }
    }
    CK(e->d_sched.alloc(e->h_sched.size()));
    CK(cudaMemcpyAsync(e->d_sched.p, e->h_sched.data(), e->h_sched.size() * sizeof(StepEntry), cudaMemcpyHostToDevice, e->cs));
    CK(e->d_prog.alloc(GR_MAX_EXPR));
    CK(cudaMemcpyAsync(e->d_prog.p, e->progs, sizeof(e->progs), cudaMemcpyHostToDevice, e->cs));

    rc = alloc_state(e);
    if (rc) return rc;
    if (s.minimum_alive > 0) {
        rc = alloc_set(e, e->ck, false);
        if (rc) return rc;
        CK(e->alive_at.alloc((size_t)kAliveSteps * 32));
    }
    const size_t N = (size_t)e->n;
    CK(e->hpos.alloc(N * e->L * e->dim));
    if (e->Lc > 0) CK(e->hcurv.alloc(N * e->Lc));
    if (e->nvol > 0 && s.volume_mode != 0 && e->Li > 0) CK(e->hvol.alloc(N * e->Li * e->nvol));
    if (e->nexpr > 0 && e->Li > 0) CK(e->hcmp.alloc(N * e->Li * e->nexpr));
    // retirement records and frozen values of retired particles (RowFill)
    CK(e->ret_rec.alloc(N));
    CK(e->frz_pos.alloc(N * e->dim));
    if (e->hvol.p) CK(e->frz_vol.alloc(N * e->nvol));
    if (e->hcmp.p) CK(e->frz_cmp.alloc(N * e->nexpr));
    if (e->Lc > 0) CK(e->frz_curv.alloc(N));

    R.rec_before.assign((size_t)R.nsteps + 1, 1);
    for (int64_t k = 0; k < R.nsteps; ++k) R.rec_before[k + 1] = R.rec_before[k] + (R.sched.steps[k].save ? 1 : 0);
    R.save_next.assign((size_t)R.nsteps + 1, R.nsteps);
    for (int64_t k = R.nsteps - 1; k >= 0; --k) R.save_next[k] = R.sched.steps[k].save ? k : R.save_next[k + 1];
    R.spl = s.steps_per_launch > 0 ? s.steps_per_launch : (int64_t)1 << 40;
    if (e->compacting && s.steps_per_launch <= 0 && R.nwin > 0)
        R.spl = std::max<int64_t>(1, R.sched.window_begin[1] - R.sched.window_begin[0]);   // one window per launch

    // window-pair layout: one load per corner returns both snapshots; launches never cross a
    // window boundary then
    e->use_pair = e->wind_dynamic && s.layout == 0;
    {
        const int rc = settle_pairs(e);
        if (rc) return rc;
    }
    e->pair_window[0] = e->pair_window[1] = -1;
    if (graph) {
        if (e->use_pair)
            for (int b = 0; b < 2; ++b) CK(e->pairbuf[b].alloc(pair_bytes(e)));
        // the curvature-record table of the full run, uploaded before the capture
        const std::vector<int32_t> t = rec_of_crec_table(e, R, R.nsteps);
        CK(e->rec_of_crec.alloc(t.size()));
        CK(cudaMemcpyAsync(e->rec_of_crec.p, t.data(), t.size() * sizeof(int32_t), cudaMemcpyHostToDevice, e->cs));
        CK(cudaStreamSynchronize(e->cs));
        CK(cudaStreamSynchronize(e->xs));   // snapshot uploads done: the graph waits on nothing outside
    }
    return GR_OK;
}

StateView view_of(gr_engine::State &S, int64_t stride) {
    StateView v;
    v.px = S.px.p; v.py = S.py.p; v.pz = S.pz.p; v.qx = S.qx.p; v.qy = S.qy.p; v.qz = S.qz.p;
    v.kx = S.kx.p; v.ky = S.ky.p; v.kz = S.kz.p; v.lx = S.lx.p; v.ly = S.ly.p; v.lz = S.lz.p;
    v.length = S.length.p; v.tc = S.tc.p; v.curv = S.curv.p; v.volc = S.volc.p; v.cmpc = S.cmpc.p;
    v.vlast = S.vlast.p;
    v.status = S.status.p; v.id = S.id.p; v.retire = S.retire.p; v.life = S.life.p; v.birth = nullptr;
    v.stride = stride;
    return v;
}

KParams make_params(gr_engine *e) {
    KParams P;
    std::memset(&P, 0, sizeof P);
    for (int d = 0; d < 3; ++d) {
        P.inv_scale[d] = e->inv_scale[d];
        P.off[d] = e->off[d];
        P.dom[d] = e->dom[d];
        P.scale[d] = e->scale[d];
    }
    P.nx = (int32_t)e->nx; P.ny = (int32_t)e->ny; P.nz = (int32_t)e->nz; P.dim = e->dim;
    P.fn[0] = (float)e->nx; P.fn[1] = (float)e->ny; P.fn[2] = (float)e->nz;
    P.pnx = (int32_t)(e->nx + 3); P.pnxy = (int32_t)((e->nx + 3) * (e->ny + 3));
    P.wind = e->wind.p; P.wind_stride = e->wind_stride;
    P.vol = e->vol.p; P.vol_plane = e->nodes;
    P.cons = e->cons.p; P.lift = e->lift.p; P.topo = e->topo.p;
    gr_engine::State &S = e->st[e->cur];
    P.px = S.px.p; P.py = S.py.p; P.pz = S.pz.p;
    P.qx = S.qx.p; P.qy = S.qy.p; P.qz = S.qz.p;
    P.kx = S.kx.p; P.ky = S.ky.p; P.kz = S.kz.p;
    P.lx = S.lx.p; P.ly = S.ly.p; P.lz = S.lz.p;
    P.status = S.status.p; P.length = S.length.p; P.tc = S.tc.p; P.curv = S.curv.p;
    P.volc = S.volc.p; P.cmpc = S.cmpc.p; P.vlast = S.vlast.p; P.vrec = e->vrec.p; P.id = S.id.p; P.life = e->has_life ? S.life.p : nullptr;
    P.n = e->n; P.n_state = e->n; P.n_total = e->n;
    P.n_dev = e->compacting ? e->d_counts.p : nullptr;
    P.hpos = e->hpos.p; P.hcurv = e->hcurv.p; P.hvol = e->hvol.p; P.hcmp = e->hcmp.p;
    P.L = e->L; P.Lc = e->Lc; P.Li = e->Li;
    P.sched = e->d_sched.p;
    const gr_settings &s = e->s;
    P.h = s.delta_t;
    P.hh = 0.5f * s.delta_t;
    P.sixth = 1.0f / 6;
    P.inv_2h = 1.0f / (2.0f * s.delta_t);
    P.inv_hh = 1.0f / (s.delta_t * s.delta_t);
    P.max_length = s.maximum_length;
    P.sphere_radius = s.sphere_radius;
    P.wind_dynamic = e->wind_dynamic;
    P.dyn_any = e->dyn_any;
    P.border_mode = e->dim == 2 ? s.border_mode : 0;
    P.curvature_mode = s.curvature_mode;
    P.abort_mode = s.abort_mode;
    P.uplift_mode = e->dim == 3 && e->has_uplift ? s.uplift_mode : 0;
    P.constants_mode = e->ncon > 0 ? s.constants_mode : 0;
    P.volume_mode = e->nvol > 0 ? s.volume_mode : 0;
    P.reverse = s.reverse ? 1 : 0;
    P.sphere = e->dim == 2 && s.sphere_radius > 0.f;
    P.topography = e->has_topo ? 1 : 0;
    P.compensated = s.compensated ? 1 : 0;
    P.filter_weights = s.filter_weights ? 1 : 0;
    P.nvol = P.volume_mode ? e->nvol : 0;
    P.ncon = P.constants_mode ? e->ncon : 0;
    P.nexpr = e->nexpr;
    P.prog = e->d_prog.p;
    P.counters = e->counters.p;
    P.alive_at = e->s.minimum_alive > 0 ? e->alive_at.p : nullptr;
    return P;
}

// One compaction / re-sort pass over the live prefix (compact.cuh).  `graph`: no host copy of
// the live count.
int compact_pass(gr_engine *e, int32_t rec_now, int32_t k_end, bool graph) {
    CompactParams C;
    std::memset(&C, 0, sizeof C);
    const int64_t N = e->n;
    C.src = view_of(e->st[e->cur], N);
    C.dst = view_of(e->st[1 - e->cur], N);
    C.ret = view_of(e->ret, N);
    if (!e->has_life) C.src.life = C.dst.life = nullptr;
    C.ret.life = nullptr;
    C.key = e->c_key.p;
    C.hist = e->c_hist.p;
    C.chunk = e->c_chunk.p;
    C.perm = e->c_perm.p;
    C.bintab = e->c_bintab.p;
    C.n_act = e->d_counts.p;
    C.n_new = e->d_counts.p + 1;
    C.n_ret = e->d_counts.p + 2;
    for (int d = 0; d < 3; ++d) {
        C.off[d] = e->off[d];
        C.inv_scale[d] = e->inv_scale[d];
    }
    C.nx = (int32_t)e->nx; C.ny = (int32_t)e->ny; C.nz = (int32_t)e->nz; C.dim = e->dim;
    C.bx = e->bx; C.by = e->by; C.bz = e->bz; C.nbx = e->nbx; C.nby = e->nby; C.nbz = e->nbz; C.nbins = e->nbins;
    const int cm = e->s.curvature_mode;
    C.nvol = (e->nvol > 0 && e->s.volume_mode != 0) ? e->nvol : 0;
    C.nexpr = e->nexpr;
    C.curv_prev = cm == 1 || cm == 3;
    C.compensated = e->s.compensated ? 1 : 0;
    C.fast_curv = cm == 2;
    C.abort_on = e->s.abort_mode != 0;
    C.curv_on = cm != 0;
    C.curv_ind = cm == 3;
    C.rec_now = rec_now;
    C.k_end = k_end;
    const int threads = 256;
    // grid-stride kernels over the device live count: a few resident waves cover any count
    const int blocks = std::min(grid_for(N, threads), 148 * 16);
    const int nchunks = (e->nbins + 1 + SCAN_CHUNK - 1) / SCAN_CHUNK;
    CK(cudaMemsetAsync(e->c_hist.p, 0, ((size_t)e->nbins + 1) * sizeof(int32_t), e->cs));
    bin_kernel<<<blocks, threads, 0, e->cs>>>(C);
    scan_chunks_kernel<<<nchunks, SCAN_CHUNK, 0, e->cs>>>(C);
    scan_top_kernel<<<1, 1024, 0, e->cs>>>(C, nchunks);
    rank_kernel<<<blocks, threads, 0, e->cs>>>(C);
    gather_kernel<<<blocks, threads, 0, e->cs>>>(C);
    commit_kernel<<<1, 1, 0, e->cs>>>(C);
    CK(cudaGetLastError());
    if (!graph) {
        CK(cudaMemcpyAsync(e->h_live, e->d_counts.p, sizeof(int32_t), cudaMemcpyDeviceToHost, e->cs));
        CK(cudaEventRecord(e->live_ready, e->cs));
    }
    e->cur = 1 - e->cur;
    e->stats.aux_launches += 6;
    return GR_OK;
}

// Final per-particle outputs of the retired store.
__global__ void finalize_retired_kernel(StateView R, const int32_t *n_ret, int abort_on, int curv_on, int32_t *status_out,
                                        float *length_out, float *tc_out) {
    const int64_t nr = *n_ret;
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < nr; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t pid = R.id[j];
        status_out[pid] = R.status[j];
        if (abort_on) length_out[pid] = R.length[j];
        if (curv_on) tc_out[pid] = R.tc[j];
    }
}

using KernelFn = void (*)(const KParams);

KernelFn pick_kernel(const gr_engine *e, const KParams &P, bool defer) {
    const bool rk4 = e->s.integrator == 1;
    const int st = e->s.storage;
    const int ft = kernel_features(P, e->use_pair, defer);
    return st == GR_STORE_BF16 ? advance_bf16(e->dim, rk4, e->use_pair, ft)
         : st == GR_STORE_F16 ? advance_f16(e->dim, rk4, e->use_pair, ft) : advance_f32(e->dim, rk4, e->use_pair, ft);
}

int block_size_for(const gr_engine *e) {
    if (e->s.block_size > 0) return e->s.block_size;
    // keep at least ~2 blocks per SM on small particle counts
    int bs = 256;
    while (bs > 32 && (e->n + bs - 1) / bs < 2 * 148) bs /= 2;
    return bs;
}

cudaEvent_t pool_event(gr_engine *e, size_t k) {
    while (e->ev_pool.size() <= k) {
        cudaEvent_t ev;
        cudaEventCreate(&ev);
        e->ev_pool.push_back(ev);
    }
    return e->ev_pool[k];
}

// Builds the window-pair buffer of window w from its two ring slots (on the compute stream).
// Packs window w's pair (ring slots w and w + 1, interleaved) into pairbuf[w & 1] on `stream`.
int pack_pair(gr_engine *e, int64_t w, cudaStream_t stream) {
    const int b = (int)(w & 1);
    const int elem = pair_elem(e);
    CK(e->pairbuf[b].alloc(pair_bytes(e)));
    const char *back = e->wind.p + (int64_t)(w % e->K) * e->wind_stride;
    const char *front = e->wind.p + (int64_t)((w + 1) % e->K) * e->wind_stride;
    const int threads = 256, blocks = grid_for(e->nodes, threads);
    if (e->dim == 3) {
        const int32_t nx = (int32_t)e->nx, ny = (int32_t)e->ny, nz = (int32_t)e->nz;
        const int b3 = grid_for(padded_pair_nodes(3, nx, ny, nz) / PACK3_UNROLL, PACK3_THREADS);
        if (elem == 16)
            pair_pack_padded_kernel<float><<<b3, PACK3_THREADS, 0, stream>>>((const float4 *)back, (const float4 *)front,
                                                                             e->pairbuf[b].p, nx, ny, nz);
        else
            pair_pack_padded_kernel<uint16_t><<<b3, PACK3_THREADS, 0, stream>>>((const uint2 *)back, (const uint2 *)front,
                                                                                e->pairbuf[b].p, nx, ny, nz);
    } else {
        const int32_t nx = (int32_t)e->nx, ny = (int32_t)e->ny;
        if (elem == 8)
            pair_pack_edge2_kernel<float><<<blocks, threads, 0, stream>>>((const float2 *)back, (const float2 *)front,
                                                                         (float4 *)e->pairbuf[b].p, nx, ny);
        else
            pair_pack_edge2_kernel<uint16_t><<<blocks, threads, 0, stream>>>(
                (const unsigned *)back, (const unsigned *)front, (uint2 *)e->pairbuf[b].p, nx, ny);
    }
    CK(cudaGetLastError());
    e->pair_window[b] = w;
    e->stats.aux_launches++;
    return GR_OK;
}

// Orders every pair packed ahead on ps before later work on cs (the end of a run, a failed run,
// the next run's first upload into a ring slot that the pack reads).
int settle_pairs(gr_engine *e) {
    for (int b = 0; b < 2; ++b)
        if (e->pair_pending[b]) {
            CK(cudaStreamWaitEvent(e->cs, e->pair_ready[b], 0));
            e->pair_pending[b] = false;
        }
    return GR_OK;
}

int ensure_pair(gr_engine *e, int64_t w) {
    const int b = (int)(w & 1);
    if (e->pair_window[b] == w) {
        if (e->pair_pending[b]) {   // packed ahead on ps
            CK(cudaStreamWaitEvent(e->cs, e->pair_ready[b], 0));
            e->pair_pending[b] = false;
        }
        return GR_OK;
    }
    return pack_pair(e, w, e->cs);
}

// Before window w's first launch: the pair of window w + 1 goes to the other buffer on ps, once
// the launches of window w - 1 (the last readers of that buffer) are done and both of its
// snapshots are in the ring, so the pack overlaps window w's launches.
int prefetch_pair(gr_engine *e, int64_t w, int64_t nwin) {
    const int64_t w1 = w + 1;
    const int b1 = (int)(w1 & 1);
    if (w1 >= nwin || e->pair_window[b1] == w1) return GR_OK;
    if (e->wind_holds[w1 % e->K] != w1 || e->wind_holds[(w1 + 1) % e->K] != w1 + 1) return GR_OK;
    CK(cudaEventRecord(e->pair_go, e->cs));
    CK(cudaStreamWaitEvent(e->ps, e->pair_go, 0));
    CK(cudaStreamWaitEvent(e->ps, e->slot_ready[w1 % e->K], 0));
    CK(cudaStreamWaitEvent(e->ps, e->slot_ready[(w1 + 1) % e->K], 0));
    const int rc = pack_pair(e, w1, e->ps);
    if (rc) return rc;
    CK(cudaEventRecord(e->pair_ready[b1], e->ps));
    e->pair_pending[b1] = true;
    return GR_OK;
}

struct RunCtx {
    gr_engine *e;
    RunPlan *R;
    KParams P;
    KernelFn fn;
    int threads;
    int64_t grid = 0;          // graph runs: persistent grid of the step kernel
    size_t ev_used = 2;        // events 0 and 1 bracket the run
    int64_t executed = 0;      // steps enqueued
    int64_t since_sort = 0;    // launches since the last compaction
    int64_t alive_known = -1;  // particles alive before the next step (-1: all of them)
    unsigned long long ps_known = 0;   // particle-steps counted before the next launch
    bool defer = false;        // volume / expression values by deferred_extras_kernel after each
                               // launch (at most one save step per launch)
};

int make_ctx(gr_engine *e, RunPlan &R, RunCtx &r) {
    r = RunCtx{};
    r.e = e;
    r.R = &R;
    r.P = make_params(e);
    // deferred volume / expression values: not in graph runs (fixed launch shapes) and only
    // where a lean variant applies
    r.defer = !R.graph && r.P.vlast != nullptr && (kernel_features(r.P, e->use_pair, true) & FT_DEFER) != 0;
    // resolved per run (a cache lookup after the first compile): expressions and settings may
    // change between runs
    e->jit_extras = nullptr;
    if (r.defer)
        e->jit_extras = jit_deferred_kernel(e->progs,
                                            JitOptions{r.P.nvol, r.P.nexpr, r.P.ncon, r.P.volume_mode, r.P.constants_mode,
                                                       r.P.curvature_mode, r.P.dyn_any},
                                            e->dim, e->jit_why);
    r.fn = pick_kernel(e, r.P, r.defer);
    r.threads = block_size_for(e);
    // some step kernels are built for smaller blocks (their launch bounds)
    cudaFuncAttributes fa{};
    CK(cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(r.fn)));
    r.threads = std::min(r.threads, fa.maxThreadsPerBlock);
    if (R.graph) {
        // one resident wave (times grid_waves) walks the live prefix with a grid-stride loop
        int per_sm = 0, sms = 0;
        CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, r.fn, r.threads, 0));
        CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->s.device));
        const int64_t waves = e->s.grid_waves > 0 ? e->s.grid_waves : 1;
        const int64_t need = (e->n + r.threads - 1) / r.threads;
        r.grid = std::max<int64_t>(1, std::min<int64_t>(need, (int64_t)std::max(1, per_sm) * sms * waves));
        r.P.grid_stride = 1;
    }
    return GR_OK;
}

int launch_steps(RunCtx &r, int64_t s0, int64_t s1, int64_t window) {
    gr_engine *e = r.e;
    KParams P = r.P;
    P.s0 = (int32_t)s0;
    P.s1 = (int32_t)s1;
    if (e->use_pair) {
        int rc = ensure_pair(e, window);
        if (rc) return rc;
        P.pair = e->pairbuf[window & 1].p;
        if (!r.R->graph && e->s.minimum_alive == 0) {
            rc = prefetch_pair(e, window, r.R->nwin);
            if (rc) return rc;
        }
    }
    if (r.R->graph) {
        r.fn<<<(unsigned)r.grid, r.threads, 0, e->cs>>>(P);
        CK(cudaGetLastError());
        e->stats.launches++;
        return GR_OK;
    }
    CK(cudaMemsetAsync(e->counters.p + 1, 0, sizeof(unsigned long long), e->cs));
    cudaEvent_t a = pool_event(e, r.ev_used++), b = pool_event(e, r.ev_used++);
    CK(cudaEventRecord(a, e->cs));
    // one thread per particle: the step kernel is not grid-strided
    const int64_t blocks = (P.n + r.threads - 1) / r.threads;
    r.fn<<<(unsigned)std::max<int64_t>(1, blocks), r.threads, 0, e->cs>>>(P);
    CK(cudaGetLastError());
    CK(cudaEventRecord(b, e->cs));
    e->stats.launches++;
    return GR_OK;
}

// Volume / expression values of a FT_DEFER run (deferred_extras_kernel): save_step >= 0 after
// the launch that ran that save step (the record's rows); else the slots with pending inputs,
// all of them or (all = false) those that retire at the compaction after step k_end.
int launch_deferred_extras(RunCtx &r, int64_t save_step, int64_t k_end, bool all) {
    gr_engine *e = r.e;
    const RunPlan &R = *r.R;
    const int32_t rec = save_step >= 0 ? R.rec_before[save_step] : -1;
    // the expression programs travel in the kernel's parameters when they fit
    ExprSet X;
    std::memset(&X, 0, sizeof X);
    int32_t total = 0;
    for (int k = 0; k < e->nexpr; ++k) total += e->progs[k].len;
    if (total <= GR_EXPR_PARAM_CODE) {
        X.in_params = 1;
        int32_t at = 0;
        for (int k = 0; k < e->nexpr; ++k) {
            X.start[k] = at;
            X.len[k] = e->progs[k].len;
            std::memcpy(X.code + at, e->progs[k].code, sizeof(Instr) * (size_t)e->progs[k].len);
            at += e->progs[k].len;
        }
    }
    const int threads = 256;
    const int blocks = grid_for(r.P.n, threads);
    if (e->jit_extras) {
        KParams P = r.P;
        int32_t a_rec = rec, a_irec = rec - 1, a_k = (int32_t)k_end, a_all = all ? 1 : 0;
        void *args[] = {&P, &a_rec, &a_irec, &a_k, &a_all};
        CK(cudaLaunchKernel(reinterpret_cast<const void *>(e->jit_extras), dim3((unsigned)blocks), dim3(threads), args, 0,
                            e->cs));
        e->stats.aux_launches++;
        e->stats.jit_launches++;
        return GR_OK;
    }
    if (e->dim == 3)
        deferred_extras_kernel<3><<<(unsigned)blocks, threads, 0, e->cs>>>(r.P, X, rec, rec - 1, (int32_t)k_end, all);
    else
        deferred_extras_kernel<2><<<(unsigned)blocks, threads, 0, e->cs>>>(r.P, X, rec, rec - 1, (int32_t)k_end, all);
    CK(cudaGetLastError());
    e->stats.aux_launches++;
    return GR_OK;
}

// After a launch that ended before step k_end: maybe retire / re-sort (compact.cuh).
int after_launch(RunCtx &r, int64_t k_end) {
    gr_engine *e = r.e;
    const RunPlan &R = *r.R;
    if (!e->compacting || k_end >= R.nsteps) return 0;
    if (++r.since_sort < (e->s.sort_interval > 0 ? e->s.sort_interval : kAutoSortInterval)) return 0;
    r.since_sort = 0;
    if (r.defer) {   // retiring particles take their final values along
        const int q = launch_deferred_extras(r, -1, k_end, false);
        if (q) return q;
    }
    int q = compact_pass(e, R.rec_before[k_end], (int32_t)k_end, R.graph);
    if (q) return q;
    const int32_t gs = r.P.grid_stride;
    r.P = make_params(e);
    r.P.grid_stride = gs;
    // live count of the last completed pass: an upper bound of the current one
    if (!R.graph) r.P.n = std::max<int64_t>(1, *(volatile int32_t *)e->h_live);
    return 0;
}

// Steps [b, t): returns 1 when MinimumAliveParticles stopped the run.
int launch_range(RunCtx &r, int64_t b, int64_t t) {
    gr_engine *e = r.e;
    const RunPlan &R = *r.R;
    if (e->s.minimum_alive > 0) {
        // The reference checks alive() before every step (tpp:973-975).  Each launch here runs
        // a whole window and counts the particles alive after every step; when the count
        // falls below the minimum inside the launch, the state saved before the launch is put
        // back and exactly the steps the reference runs are launched again.
        const long long minimum = e->s.minimum_alive;
        for (int64_t k = b; k < t;) {
            const long long alive = r.alive_known < 0 ? e->n : r.alive_known;
            if (alive < minimum) return 1;
            int64_t k1 = std::min({t, k + R.spl, k + kAliveSteps});
            const int64_t w = R.sched.steps[k].window;
            if (e->use_pair) k1 = std::min(k1, R.sched.window_begin[w + 1]);
            const int64_t L = k1 - k;
            gr_engine::State &S = e->st[e->cur];
            const int64_t live = r.P.n;   // upper bound of the live prefix
            if (L > 1) {
                const int q = copy_state(e, e->ck, S, live);
                if (q) return q;
            }
            CK(cudaMemsetAsync(e->alive_at.p, 0, (size_t)L * 32 * sizeof(unsigned), e->cs));
            int q = launch_steps(r, k, k1, w);
            if (q) return q;
            e->h_alive.resize((size_t)L * 32);
            CK(cudaMemcpyAsync(e->h_alive.data(), e->alive_at.p, (size_t)L * 32 * sizeof(unsigned),
                               cudaMemcpyDeviceToHost, e->cs));
            CK(cudaMemcpyAsync(e->h_counters, e->counters.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                               e->cs));
            CK(cudaStreamSynchronize(e->cs));
            auto alive_after = [&](int64_t j) {   // alive after step k + j
                long long a = 0;
                for (int h = 0; h < 32; ++h) a += e->h_alive[(size_t)j * 32 + h];
                return a;
            };
            int64_t stop = -1;   // first step of the launch the reference does not run
            for (int64_t j = 1; j < L && stop < 0; ++j)
                if (alive_after(j - 1) < minimum) stop = k + j;
            if (stop >= 0) {
                // roll back, then run steps [k, stop) only
                q = copy_state(e, S, e->ck, live);
                if (q) return q;
                CK(cudaMemcpyAsync(e->counters.p, &r.ps_known, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                   e->cs));
                q = launch_steps(r, k, stop, w);
                if (q) return q;
                CK(cudaStreamSynchronize(e->cs));   // the copy above reads r.ps_known
                r.executed += stop - k;
                return 1;
            }
            r.alive_known = alive_after(L - 1);
            r.ps_known = e->h_counters[0];
            r.executed += L;
            q = after_launch(r, k1);
            if (q) return q;
            k = k1;
        }
        return 0;
    }
    for (int64_t k = b; k < t;) {
        int64_t k1 = std::min(t, k + R.spl);
        const int64_t w = R.sched.steps[k].window;
        if (e->use_pair) k1 = std::min(k1, R.sched.window_begin[w + 1]);   // one window per launch
        if (r.defer && R.save_next[k] < R.nsteps)
            k1 = std::min(k1, R.save_next[R.save_next[k] + 1]);            // and one save step
        int q = launch_steps(r, k, k1, w);
        if (q) return q;
        if (r.defer && R.save_next[k] < k1) {
            q = launch_deferred_extras(r, R.save_next[k], k1, false);
            if (q) return q;
        }
        q = after_launch(r, k1);
        if (q) return q;
        k = k1;
    }
    r.executed += t - b;
    return 0;
}

// ---------------------------------------------------------------- result streaming

// Row bytes per particle below which a streamed copy waits for more records: pitched DMAs of
// short rows run well below the link rate (about 38 GB/s at 240 B, 52 GB/s at 600 B on B200).
constexpr int64_t kStreamRowBytes = 256;

// Checks the destinations against this run's history and turns streaming on for it.
int stream_begin(gr_engine *e, const RunPlan &R) {
    e->dest_run = e->dest_during = false;
    e->streamed = 0;
    if (!e->dest_set || R.graph) return GR_OK;
    const gr_result_destinations &d = e->dest;
    const size_t n = (size_t)e->n;
    if (d.positions) {
        if (d.records_capacity < e->L)
            return USER_ERR("Result destinations hold %lld records per particle; the run writes %lld. >",
                            (long long)d.records_capacity, (long long)e->L);
        if (!pinned_range(d.positions, n * (size_t)d.records_capacity * e->dim * sizeof(float)))
            return USER_ERR("Result destinations must be page-locked host memory. >");
    }
    auto check_info = [&](const float *a) -> int {
        if (!a || e->Li == 0) return GR_OK;
        if (d.info_capacity < e->Li)
            return USER_ERR("Result destinations hold %lld info records per particle; the run writes %lld. >",
                            (long long)d.info_capacity, (long long)e->Li);
        if (!pinned_range(a, n * (size_t)std::max<int64_t>(d.info_capacity, 1) * sizeof(float)))
            return USER_ERR("Result destinations must be page-locked host memory. >");
        return GR_OK;
    };
    for (int k = 0; k < (e->s.volume_mode != 0 ? e->nvol : 0); ++k) {
        const int rc = check_info(d.volume_info[k]);
        if (rc) return rc;
    }
    for (int k = 0; k < e->nexpr; ++k) {
        const int rc = check_info(d.compute_info[k]);
        if (rc) return rc;
    }
    if (!e->ds) CK(cudaStreamCreateWithFlags(&e->ds, cudaStreamNonBlocking));
    if (!e->ds_ev) CK(cudaEventCreateWithFlags(&e->ds_ev, cudaEventDisableTiming));
    e->dest_run = true;
    e->dest_during = e->s.minimum_alive == 0;
    return GR_OK;
}

// Retirement records and frozen values of the retired store so far, on the step stream.
int note_retired(gr_engine *e) {
    const StateView Rv = view_of(e->ret, e->n);
    const int nvol = e->hvol.p ? e->nvol : 0, nexpr = e->hcmp.p ? e->nexpr : 0;
    note_retired_kernel<<<grid_for(e->n, 256), 256, 0, e->cs>>>(Rv, e->d_counts.p + 2, e->dim, nvol, nexpr,
                                                               e->Lc > 0 ? 1 : 0, e->n, e->ret_rec.p, e->frz_pos.p,
                                                               e->frz_vol.p, e->frz_cmp.p, e->frz_curv.p);
    CK(cudaGetLastError());
    e->stats.aux_launches++;
    return GR_OK;
}

// The RowFill of a record-major quantity whose frozen values are frz (no substitution without a
// retired store).
RowFill row_fill(const gr_engine *e, const float *frz, int32_t rec_offset, const int32_t *rec_of_row) {
    RowFill f{};
    if (e->compacting && e->ret_rec.p) {
        f.ret = e->ret_rec.p;
        f.frz = frz;
        f.rec_offset = rec_offset;
        f.rec_of_row = rec_of_row;
    }
    return f;
}

// Record-major history -> particle-major rows on the device: records [r0, r1) of particles
// [p0, p1) of a quantity with D floats per particle (records_to_rows_kernel), on `st`.
int launch_records_to_rows(gr_engine *e, cudaStream_t st, const float *src, int64_t n, int D, int32_t r0,
                           int32_t r1, int64_t p0, int64_t p1, float *dst, const RowFill &fill) {
    constexpr int32_t kRowsPerLaunch = 32 * 65535;   // the grid's y extent
    for (int32_t a = r0; a < r1; a += kRowsPerLaunch) {
        const int32_t b = std::min(r1, a + kRowsPerLaunch);
        // each launch covers records [a, b) of the destination rows sized for [r0, r1)
        const dim3 grid((unsigned)((p1 - p0 + 31) / 32), (unsigned)((b - a + 31) / 32));
        float *d = dst + (int64_t)(a - r0) * D;
        const int32_t nr = r1 - r0;
        if (D == 1) records_to_rows_kernel<1><<<grid, 256, 0, st>>>(src, n, a, b, p0, p1, d, nr, fill);
        else if (D == 2) records_to_rows_kernel<2><<<grid, 256, 0, st>>>(src, n, a, b, p0, p1, d, nr, fill);
        else records_to_rows_kernel<3><<<grid, 256, 0, st>>>(src, n, a, b, p0, p1, d, nr, fill);
        CK(cudaGetLastError());
        e->stats.aux_launches++;
    }
    return GR_OK;
}

// Particles per staging chunk for particle-major rows of `row_floats` floats.
int64_t stage_particles(int64_t n, int64_t row_floats) {
    constexpr int64_t kStageBytes = int64_t(256) << 20;
    return std::max<int64_t>(1, std::min<int64_t>(n, kStageBytes / std::max<int64_t>(1, row_floats * 4)));
}

// Copies records [e->streamed, r1) of every particle (and their volume / compute records) into
// the destinations on the copy-out stream, behind everything already on the step stream.
// Particles retired so far get those records filled first; particles still in the live set
// wrote them in the step kernel.
int stream_records(RunCtx &r, int32_t r1) {
    gr_engine *e = r.e;
    const int32_t r0 = e->streamed;
    if (r1 <= r0 || e->n == 0) return GR_OK;
    if (e->compacting) {
        const int rc = note_retired(e);
        if (rc) return rc;
    }
    CK(cudaEventRecord(e->ds_ev, e->cs));
    CK(cudaStreamWaitEvent(e->ds, e->ds_ev, 0));
    const gr_result_destinations &d = e->dest;
    const int64_t n = e->n;
    // records [a, b) of a record-major quantity (D floats per particle) into host rows of `dpitch`
    // floats, from column a * D: chunks of particles transposed into the streaming stage, each
    // followed by one pitched DMA (both on the copy-out stream, so a chunk's DMA ends before the
    // next transpose reuses the stage)
    auto stream_rows = [&](float *dst, int64_t dpitch, const float *src, int D, int32_t a, int32_t b,
                           const RowFill &fill) -> int {
        const int64_t w = (int64_t)(b - a) * D;
        const int64_t cp = stage_particles(n, w);
        if ((size_t)(cp * w) > e->sstage.count) {
            CK(cudaStreamSynchronize(e->ds));   // earlier DMAs may still read the old stage
            CK(e->sstage.alloc((size_t)(cp * w)));
        }
        for (int64_t p0 = 0; p0 < n; p0 += cp) {
            const int64_t p1 = std::min(n, p0 + cp);
            const int rc = launch_records_to_rows(e, e->ds, src, n, D, a, b, p0, p1, e->sstage.p, fill);
            if (rc) return rc;
            CK(cudaMemcpy2DAsync(dst + p0 * dpitch + (int64_t)a * D, (size_t)dpitch * sizeof(float), e->sstage.p,
                                 (size_t)w * sizeof(float), (size_t)w * sizeof(float), (size_t)(p1 - p0),
                                 cudaMemcpyDeviceToHost, e->ds));
        }
        e->stats.d2h_bytes += w * n * (int64_t)sizeof(float);
        return GR_OK;
    };
    if (d.positions) {
        const int rc = stream_rows(d.positions, d.records_capacity * e->dim, e->hpos.p, e->dim, r0, r1,
                                   row_fill(e, e->frz_pos.p, 0, nullptr));
        if (rc) return rc;
    }
    // info record i belongs to position record i + 1
    const int32_t i0 = std::max(r0 - 1, 0), i1 = r1 - 1;
    if (i1 > i0) {
        // info record i belongs to position record i + 1
        auto copy_info = [&](float *dst, const float *src, const float *frz) -> int {
            if (!dst) return GR_OK;
            return stream_rows(dst, d.info_capacity, src, 1, i0, i1, row_fill(e, frz, 1, nullptr));
        };
        for (int k = 0; k < (e->s.volume_mode != 0 ? e->nvol : 0); ++k) {
            const int rc = copy_info(d.volume_info[k], e->hvol.p + (size_t)k * n * e->Li, e->frz_vol.p + (size_t)k * n);
            if (rc) return rc;
        }
        for (int k = 0; k < e->nexpr; ++k) {
            const int rc = copy_info(d.compute_info[k], e->hcmp.p + (size_t)k * n * e->Li, e->frz_cmp.p + (size_t)k * n);
            if (rc) return rc;
        }
    }
    e->streamed = r1;
    return GR_OK;
}

// During the run: streams the records complete after the steps enqueued so far once they fill
// rows of kStreamRowBytes.
int stream_progress(RunCtx &r) {
    gr_engine *e = r.e;
    if (!e->dest_during) return GR_OK;
    const int32_t done = r.R->rec_before[(size_t)r.executed];
    if ((int64_t)(done - e->streamed) * e->dim * (int64_t)sizeof(float) < kStreamRowBytes) return GR_OK;
    return stream_records(r, done);
}

// Record counts after `executed` steps, including the SaveInterval == 0 final record.
struct RecordCounts {
    int64_t rec = 1, crec = 0, irec = 0;
};

RecordCounts count_records(const RunPlan &R, int64_t executed) {
    RecordCounts c;
    for (int64_t k = 0; k < executed; ++k)
        if (R.sched.steps[k].save) {
            ++c.rec;
            ++c.irec;
            if (R.sched.steps[k].time_pos) ++c.crec;
        }
    return c;
}

// After the step loop: the SaveInterval == 0 final record, final per-particle outputs, and the
// records of retired particles.  Graph runs upload the fill-forward table beforehand.
int run_tail(RunCtx &r, RecordCounts &c) {
    gr_engine *e = r.e;
    const RunPlan &R = *r.R;
    const gr_settings &s = e->s;
    const int64_t executed = r.executed;
    c = count_records(R, executed);
    KParams P = r.P;
    if (r.defer) {   // pending volume / expression values into the state arrays
        const int q = launch_deferred_extras(r, -1, executed, true);
        if (q) return q;
    }
    if (s.save_interval == 0) {
        const bool tpos = executed > 0;   // data.Time > 0 after at least one step
        if (e->dim == 3)
            save_state_kernel<3><<<grid_for(e->n, 256), 256, 0, e->cs>>>(P, (int32_t)c.rec, (int32_t)c.crec, (int32_t)c.irec, tpos);
        else
            save_state_kernel<2><<<grid_for(e->n, 256), 256, 0, e->cs>>>(P, (int32_t)c.rec, (int32_t)c.crec, (int32_t)c.irec, tpos);
        CK(cudaGetLastError());
        ++c.rec;
        ++c.irec;
        if (tpos) ++c.crec;
        e->stats.aux_launches++;
    }
    finalize_kernel<<<grid_for(e->n, 256), 256, 0, e->cs>>>(P, e->out_status.p, e->out_length.p, e->out_tc.p);
    CK(cudaGetLastError());
    e->stats.aux_launches++;
    if (e->compacting) {
        // retired particles: their later records repeat the frozen state, substituted when the
        // history is read (RowFill)
        std::vector<int32_t> t;
        if (!R.graph) {
            t = rec_of_crec_table(e, R, executed);
            CK(e->rec_of_crec.alloc(t.size()));
            CK(cudaMemcpyAsync(e->rec_of_crec.p, t.data(), t.size() * sizeof(int32_t), cudaMemcpyHostToDevice, e->cs));
        }
        const int rc = note_retired(e);
        if (rc) return rc;
        const StateView Rv = view_of(e->ret, e->n);
        finalize_retired_kernel<<<grid_for(e->n, 256), 256, 0, e->cs>>>(Rv, e->d_counts.p + 2, s.abort_mode != 0,
                                                                         s.curvature_mode != 0, e->out_status.p,
                                                                         e->out_length.p, e->out_tc.p);
        CK(cudaGetLastError());
        if (!R.graph) CK(cudaStreamSynchronize(e->cs));   // the host table t is read by the copy above
        e->stats.aux_launches++;
    }
    return GR_OK;
}

// After the device work finished: counters, timings and result sizes.
int run_collect(gr_engine *e, const RunPlan &R, int64_t executed, int64_t windows_run, const RecordCounts &c,
                size_t ev_used) {
    const gr_settings &s = e->s;
    CK(cudaMemcpyAsync(e->h_counters, e->counters.p, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, e->cs));
    CK(cudaStreamSynchronize(e->cs));
    if (ev_used >= 2) {
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, e->ev_pool[0], e->ev_pool[1]));
        e->stats.run_ms = ms;
        double kms = 0.0;
        for (size_t k = 2; k + 1 < ev_used; k += 2) {
            float t = 0.f;
            CK(cudaEventElapsedTime(&t, e->ev_pool[k], e->ev_pool[k + 1]));
            kms += t;
        }
        e->stats.kernel_ms = kms;
    }
    e->stats.particle_steps = (int64_t)e->h_counters[0];
    (void)R;
    e->info.n = e->n;
    e->info.dim = e->dim;
    e->info.records = c.rec;
    e->info.curvature_records = s.curvature_mode == 3 ? c.crec : 0;
    e->info.info_records = c.irec;
    e->info.steps = executed;
    e->info.windows = windows_run;
    e->info.particle_steps = (int64_t)e->h_counters[0];
    e->info.n_volumes = s.volume_mode != 0 ? e->nvol : 0;
    e->info.n_expressions = e->nexpr;
    e->have_result = true;
    return GR_OK;
}

int call_loader(gr_engine *e, gr_loader_fn loader, void *user, int64_t snapshot, int &result) {
    if (!loader) {
        result = 0;
        return GR_OK;
    }
    result = loader(user, e, snapshot);
    if (result < 0) {
        if (g_last_error.empty()) g_last_error = "ERROR < RUNTIME | the loader callback failed >";
        return GR_ERR_CALLBACK;
    }
    if (result > 0) {
        const int slot = (int)(snapshot % e->K);
        if (e->wind_dynamic && e->wind_holds[slot] != snapshot)
            return fail(GR_ERR_USER, "ERROR < USER INPUT | The loader did not provide windfield snapshot %lld. >",
                        (long long)snapshot);
    }
    return GR_OK;
}

}  // namespace

extern "C" int gr_run(gr_engine *e, gr_loader_fn loader, void *user) {
    if (!e) return USER_ERR("null engine >");
    if (!e->plan) e->plan = std::make_unique<RunPlan>();
    RunPlan &R = *e->plan;
    int rc = run_prepare(e, R, false);
    if (rc) return rc;
    rc = reset_state(e);
    if (rc) return rc;
    const gr_settings &s = e->s;

    cudaEvent_t run_a = pool_event(e, 0), run_b = pool_event(e, 1);
    RunCtx r;
    rc = make_ctx(e, R, r);
    if (rc) return rc;
    rc = stream_begin(e, R);
    if (rc) return rc;
    CK(cudaEventRecord(run_a, e->cs));
    // the first windows read snapshots already uploaded
    for (int k = 0; k < e->K; ++k)
        if (e->wind_holds[k] >= 0 || e->vol_holds[k] >= 0 || e->cons_holds[k] >= 0 || e->lift_holds[k] >= 0)
            CK(cudaStreamWaitEvent(e->cs, e->slot_ready[k], 0));

    const int64_t nwin = R.nwin;
    const int64_t gmax = std::max(1, e->K - 1);
    int64_t windows_run = 0;
    bool stop = false;
    int64_t w = 0;
    while (w < nwin && !stop) {
        int64_t g_end = w + 1;
        bool exhausted = false;
        // windows w .. g_end-1 run in one group; their snapshots must all fit in the ring
        while (g_end < nwin && g_end - w < gmax && s.minimum_alive == 0 && e->dyn_any) {
            int res = 0;
            rc = call_loader(e, loader, user, g_end + 1, res);   // the loader step after window g_end-1
            if (rc) return rc;
            if (res == 0) { exhausted = true; break; }
            CK(cudaStreamWaitEvent(e->cs, e->slot_ready[(g_end + 1) % e->K], 0));
            ++g_end;
        }
        for (int64_t k = w; k < g_end + (e->dyn_any ? 1 : 0) && k <= w + e->K; ++k)
            CK(cudaStreamWaitEvent(e->cs, e->slot_ready[k % e->K], 0));
        const int q = launch_range(r, R.sched.window_begin[w], R.sched.window_begin[g_end]);
        if (q < 0) return q;
        windows_run = g_end;
        // slots read by this group become free once it has run
        for (int64_t k = w; k <= g_end && k - w < e->K; ++k) {
            CK(cudaEventRecord(e->slot_free[k % e->K], e->cs));
            e->slot_used[k % e->K] = true;
        }
        const bool alive_abort = q == 1;
        rc = stream_progress(r);
        if (rc) return rc;
        if (exhausted) break;
        if (e->dyn_any) {
            int res = 0;
            rc = call_loader(e, loader, user, g_end + 1, res);   // loader step after window g_end-1
            if (rc) return rc;
            if (res == 0 || alive_abort) break;
            CK(cudaStreamWaitEvent(e->cs, e->slot_ready[(g_end + 1) % e->K], 0));
        } else {
            break;
        }
        if (alive_abort) stop = true;
        w = g_end;
    }

    RecordCounts c;
    rc = run_tail(r, c);
    if (rc) return rc;
    rc = settle_pairs(e);   // a pair packed ahead for a window that did not run
    if (rc) return rc;
    if (e->dest_run) {
        // the rest of the records; the run ends when they are in host memory
        rc = stream_records(r, (int32_t)c.rec);
        if (rc) return rc;
        CK(cudaEventRecord(e->ds_ev, e->ds));
        CK(cudaStreamWaitEvent(e->cs, e->ds_ev, 0));
    }
    CK(cudaEventRecord(run_b, e->cs));
    return run_collect(e, R, r.executed, windows_run, c, r.ev_used);
}

extern "C" int gr_set_result_destinations(gr_engine *e, const gr_result_destinations *dest) {
    if (!e) return USER_ERR("null engine >");
    if (!dest) {
        e->dest = gr_result_destinations{};
        e->dest_set = false;
        return GR_OK;
    }
    if (dest->records_capacity < 0 || dest->info_capacity < 0) return USER_ERR("negative capacity >");
    e->dest = *dest;
    e->dest_set = true;
    return GR_OK;
}

// ------------------------------------------------------------------ graph runs (batch.cu)

namespace granite_b200 {

int graph_prepare(gr_engine *e) {
    if (!e) return USER_ERR("null engine >");
    if (!e->plan) e->plan = std::make_unique<RunPlan>();
    return run_prepare(e, *e->plan, true);
}

int graph_enqueue(gr_engine *e) {
    RunPlan &R = *e->plan;
    e->pair_window[0] = e->pair_window[1] = -1;   // every window pair is packed inside the run
    int rc = reset_state(e);
    if (rc) return rc;
    RunCtx r;
    rc = make_ctx(e, R, r);
    if (rc) return rc;
    rc = launch_range(r, 0, R.nsteps);
    if (rc < 0) return rc;
    RecordCounts c;
    rc = run_tail(r, c);
    if (rc) return rc;
    e->graph_executed = r.executed;
    e->graph_records = c.rec;
    return GR_OK;
}

int graph_collect(gr_engine *e) {
    const RunPlan &R = *e->plan;
    RecordCounts c = count_records(R, e->graph_executed);
    if (e->s.save_interval == 0) {
        ++c.rec;
        ++c.irec;
        if (e->graph_executed > 0) ++c.crec;
    }
    const int64_t launches = e->stats.launches, aux = e->stats.aux_launches;
    const int rc = run_collect(e, R, e->graph_executed, R.nwin, c, 0);
    e->stats.launches = launches;
    e->stats.aux_launches = aux;
    return rc;
}

cudaStream_t engine_stream(gr_engine *e) { return e->cs; }
int engine_device(const gr_engine *e) { return e->s.device; }
uint64_t engine_generation(const gr_engine *e) { return e->gen; }
int64_t engine_launches(const gr_engine *e, int64_t *aux) {
    if (aux) *aux = e->stats.aux_launches;
    return e->stats.launches;
}
int64_t engine_particle_steps(const gr_engine *e) { return e->stats.particle_steps; }

}  // namespace granite_b200

extern "C" {

int gr_result_info_get(gr_engine *e, gr_result_info *out) {
    if (!e || !out) return USER_ERR("null argument >");
    if (!e->have_result) return USER_ERR("No result: run() has not completed. >");
    *out = e->info;
    return GR_OK;
}

int gr_stats_get(gr_engine *e, gr_stats *out) {
    if (!e || !out) return USER_ERR("null argument >");
    *out = e->stats;
    return GR_OK;
}

static int fetch_rows(gr_engine *e, void *out, int64_t capacity, const void *src, int64_t rows, int64_t row_used,
                      int64_t row_stride, size_t elem) {
    if (!e || !out) return USER_ERR("null argument >");
    if (!e->have_result) return USER_ERR("No result: run() has not completed. >");
    if (capacity < rows * row_used) return USER_ERR("Output buffer too small. >");
    if (rows == 0 || row_used == 0) return GR_OK;
    int rc = set_device(e);
    if (rc) return rc;
    const size_t row_bytes = (size_t)row_used * elem, total = row_bytes * (size_t)rows;
    e->stats.d2h_bytes += (int64_t)total;
    if (pinned_range(out, total)) {
        // page-locked destination: one DMA, no staging
        CK(cudaMemcpy2DAsync(out, row_bytes, src, row_stride * elem, row_bytes, rows, cudaMemcpyDeviceToHost, e->cs));
        CK(cudaStreamSynchronize(e->cs));
        return GR_OK;
    }
    // up to 64 MB per bounce buffer; results from 8 MB on go through them, so the host copies
    // (and the first-touch page faults of a fresh destination) run on the copy threads
    constexpr size_t kBounce = size_t(64) << 20, kBounceFrom = size_t(8) << 20;
    if (total < kBounceFrom || row_bytes > kBounce) {
        CK(cudaMemcpy2D(out, row_bytes, src, row_stride * elem, row_bytes, rows, cudaMemcpyDeviceToHost));
        return GR_OK;
    }
    // large results: DMA into two pinned bounce buffers, each emptied by a parallel host copy
    // while the other fills
    const size_t chunk = std::min(kBounce, total);
    for (auto &b : e->bounce) {
        if (b.bytes < chunk) {
            if (b.p) gr_host_free(b.p);
            b.p = nullptr;
            b.bytes = 0;
            if (gr_host_alloc((int64_t)chunk, &b.p) != GR_OK) return GR_ERR_RUNTIME;
            b.bytes = chunk;
        }
        if (!b.done) CK(cudaEventCreateWithFlags(&b.done, cudaEventDisableTiming));
    }
    const int64_t rows_per = (int64_t)(std::min(e->bounce[0].bytes, e->bounce[1].bytes) / row_bytes);
    const char *s8 = static_cast<const char *>(src);
    char *d8 = static_cast<char *>(out);
    int64_t prev_rows = 0, prev_row0 = 0;
    int j = 0;
    for (int64_t r0 = 0; r0 < rows; r0 += rows_per, j ^= 1) {
        const int64_t nr = std::min(rows_per, rows - r0);
        CK(cudaMemcpy2DAsync(e->bounce[j].p, row_bytes, s8 + (size_t)r0 * row_stride * elem, row_stride * elem,
                             row_bytes, nr, cudaMemcpyDeviceToHost, e->cs));
        CK(cudaEventRecord(e->bounce[j].done, e->cs));
        if (prev_rows) {
            CK(cudaEventSynchronize(e->bounce[j ^ 1].done));
            parallel_memcpy(d8 + (size_t)prev_row0 * row_bytes, e->bounce[j ^ 1].p, (size_t)prev_rows * row_bytes);
        }
        prev_rows = nr;
        prev_row0 = r0;
    }
    CK(cudaEventSynchronize(e->bounce[j ^ 1].done));
    parallel_memcpy(d8 + (size_t)prev_row0 * row_bytes, e->bounce[j ^ 1].p, (size_t)prev_rows * row_bytes);
    return GR_OK;
}

// Records [r0, r1) of a record-major quantity (D floats per particle) into particle-major host
// rows of (r1 - r0) * D floats: chunks of particles transposed on the device into the staging
// buffer (retired particles' frozen values substituted, RowFill), each fetched like any device
// rows.
static int fetch_records(gr_engine *e, float *out, int64_t cap, const float *src, int D, int64_t r0, int64_t r1,
                         const RowFill &fill) {
    if (!e || !out) return USER_ERR("null argument >");
    if (!e->have_result) return USER_ERR("No result: run() has not completed. >");
    const int64_t n = e->n, w = (r1 - r0) * D;
    if (cap < n * w) return USER_ERR("Output buffer too small. >");
    if (n == 0 || w == 0) return GR_OK;
    int rc = set_device(e);
    if (rc) return rc;
    const int64_t cp = stage_particles(n, w);
    CK(e->stage.alloc((size_t)(cp * w)));
    for (int64_t p0 = 0; p0 < n; p0 += cp) {
        const int64_t p1 = std::min(n, p0 + cp);
        rc = launch_records_to_rows(e, e->cs, src, n, D, (int32_t)r0, (int32_t)r1, p0, p1, e->stage.p, fill);
        if (rc) return rc;
        CK(cudaStreamSynchronize(e->cs));
        rc = fetch_rows(e, out + p0 * w, (p1 - p0) * w, e->stage.p, p1 - p0, w, w, sizeof(float));
        if (rc) return rc;
    }
    return GR_OK;
}

int gr_fetch_positions(gr_engine *e, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    return fetch_records(e, out, cap, e->hpos.p, e->dim, 0, e->info.records, row_fill(e, e->frz_pos.p, 0, nullptr));
}

int gr_fetch_final_positions(gr_engine *e, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    if (!e->have_result) return USER_ERR("No result: run() has not completed. >");
    // the last record's row
    return fetch_records(e, out, cap, e->hpos.p, e->dim, e->info.records - 1, e->info.records,
                         row_fill(e, e->frz_pos.p, 0, nullptr));
}

int gr_fetch_status(gr_engine *e, int32_t *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    return fetch_rows(e, out, cap, e->out_status.p, 1, e->n, e->n, sizeof(int32_t));
}

int gr_fetch_lengths(gr_engine *e, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    if (e->s.abort_mode == 0) return GR_OK;
    return fetch_rows(e, out, cap, e->out_length.p, 1, e->n, e->n, sizeof(float));
}

int gr_fetch_total_curvature(gr_engine *e, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    if (e->s.curvature_mode == 0) return GR_OK;
    return fetch_rows(e, out, cap, e->out_tc.p, 1, e->n, e->n, sizeof(float));
}

int gr_fetch_curvatures(gr_engine *e, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    if (e->info.curvature_records == 0) return GR_OK;
    return fetch_records(e, out, cap, e->hcurv.p, 1, 0, e->info.curvature_records,
                         row_fill(e, e->frz_curv.p, 0, e->rec_of_crec.p));
}

int gr_fetch_volume_info(gr_engine *e, int32_t index, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    if (index < 0 || index >= e->info.n_volumes) return USER_ERR("TrajectorySet: Volume with given key does not exist! >");
    if (e->info.info_records == 0) return GR_OK;
    return fetch_records(e, out, cap, e->hvol.p + (int64_t)index * e->n * e->Li, 1, 0, e->info.info_records,
                         row_fill(e, e->frz_vol.p + (int64_t)index * e->n, 1, nullptr));
}

int gr_fetch_compute_info(gr_engine *e, int32_t index, float *out, int64_t cap) {
    if (!e) return USER_ERR("null engine >");
    if (index < 0 || index >= e->info.n_expressions) return USER_ERR("TrajectorySet: Volume with given id does not exist! >");
    if (e->info.info_records == 0) return GR_OK;
    return fetch_records(e, out, cap, e->hcmp.p + (int64_t)index * e->n * e->Li, 1, 0, e->info.info_records,
                         row_fill(e, e->frz_cmp.p + (int64_t)index * e->n, 1, nullptr));
}

}  // extern "C"

// ------------------------------------------------------------------ autotuner

namespace {

// Times one configuration over the first `steps` steps (graph launch shapes, not captured);
// the faster of two runs, so lazy module loading does not count.
int tune_trial(gr_engine *e, const gr_settings &cfg, int32_t steps, double &rate) {
    e->s = cfg;
    e->step_cap = steps;
    rate = 0.0;
    cudaEvent_t a = pool_event(e, 0), b = pool_event(e, 1);
    for (int rep = 0; rep < 2; ++rep) {
        int rc = granite_b200::graph_prepare(e);
        if (rc) return rc;
        CK(cudaEventRecord(a, e->cs));
        rc = granite_b200::graph_enqueue(e);
        if (rc) return rc;
        CK(cudaEventRecord(b, e->cs));
        CK(cudaStreamSynchronize(e->cs));
        float ms = 0.f;
        CK(cudaEventElapsedTime(&ms, a, b));
        rc = granite_b200::graph_collect(e);
        if (rc) return rc;
        if (ms > 0.f) rate = std::max(rate, (double)e->stats.particle_steps / (ms * 1e-3));
    }
    return GR_OK;
}

}  // namespace

extern "C" int gr_tune(gr_engine *e, int32_t trial_steps, gr_tune_result *out) {
    if (!e) return USER_ERR("null engine >");
    if (e->s.minimum_alive > 0)
        return USER_ERR("MinimumAliveParticles needs host decisions between steps; it cannot run in a graph. >");
    const int32_t steps = trial_steps > 0 ? trial_steps : 40;
    const gr_settings base = e->s;
    gr_settings cur = base;
    if (cur.block_size <= 0) cur.block_size = 256;
    if (cur.sort_interval <= 0) cur.sort_interval = 4;
    if (cur.grid_waves <= 0) cur.grid_waves = 1;
    int trials = 0;
    double best = 0.0;
    int rc = tune_trial(e, cur, steps, best);
    ++trials;
    // coordinate descent: layout, block size, sort interval, grid waves
    auto consider = [&](gr_settings c) -> int {
        double r = 0.0;
        const int q = tune_trial(e, c, steps, r);
        ++trials;
        if (q) return q;
        if (r > best * 1.01) {
            best = r;
            cur = c;
        }
        return 0;
    };
    if (!rc && e->wind_dynamic) {
        gr_settings c = cur;
        c.layout = cur.layout == 0 ? 1 : 0;
        rc = consider(c);
    }
    for (int bs : {64, 128, 256})
        if (!rc && bs != cur.block_size) {
            gr_settings c = cur;
            c.block_size = bs;
            rc = consider(c);
        }
    for (int si : {1, 2, 4, 8})
        if (!rc && si != cur.sort_interval) {
            gr_settings c = cur;
            c.sort_interval = si;
            rc = consider(c);
        }
    for (int gw : {1, 2, 4})
        if (!rc && gw != cur.grid_waves) {
            gr_settings c = cur;
            c.grid_waves = gw;
            rc = consider(c);
        }
    e->step_cap = 0;
    ++e->gen;
    e->have_result = false;
    if (rc) {
        e->s = base;
        return rc;
    }
    e->s = cur;
    if (out) {
        out->layout = cur.layout;
        out->block_size = cur.block_size;
        out->sort_interval = cur.sort_interval;
        out->grid_waves = cur.grid_waves;
        out->particle_steps_per_s = best;
        out->trials = trials;
    }
    return GR_OK;
}
