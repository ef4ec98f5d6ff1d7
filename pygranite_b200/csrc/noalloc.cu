// noalloc.cu — gr_advance_noalloc: advancing particles without allocating device memory.
//
// Some callers cannot call cudaMalloc: plug-in hosts whose device memory belongs to their own
// pool allocator (a cudaMalloc there would go around the host's accounting and limits), and
// real-time loops that forbid allocation after start-up (an allocation may synchronise the
// device or take an unbounded time).  This entry point gives them the plain integrator (Euler
// or RK4 between two snapshots, the border checks and abort codes) on buffers they own.  Its
// only scratch, the per-step time weights and two counters, is the file-scope array below:
// every GPU that loads the library keeps these GR_NOALLOC_SCRATCH_BYTES until the process
// exits, and every call shares them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/granite_b200.h"
#include "granite_kernels.cuh"

namespace granite_b200 {
void set_last_error(const char *msg);   // engine.cu
}

using namespace granite_b200;

namespace {

struct NoAllocScratch {
    StepEntry sched[GR_NOALLOC_MAX_STEPS];
    unsigned long long counters[2];   // [0] particle-steps, [1] alive after the call
};

static_assert(sizeof(NoAllocScratch) == GR_NOALLOC_SCRATCH_BYTES, "scratch size stated in granite_b200.h");

static __device__ __align__(256) NoAllocScratch g_scratch;

constexpr int MAX_DEVICES = 64;
std::mutex g_mutex;
NoAllocScratch *g_scratch_ptr[MAX_DEVICES] = {};   // device address of g_scratch, per device

int err(int code, const char *msg) {
    set_last_error(msg);   // reported by gr_last_error()
    return code;
}

// Time weights of `steps` steps from time_start, with the float32 arithmetic of
// TrajectoryIntegrator.tpp:126-144 (the file is built with --fmad=false, so nothing is
// contracted).  The time accumulator T = T + h is a dependent chain: thread 0 walks it and
// parks each step's start time in t0; then the block turns the start times into the weights.
__global__ void __launch_bounds__(256) noalloc_schedule_kernel(NoAllocScratch *S, float time_back, float time_front,
                                                               float time_start, float h, int32_t steps) {
    if (threadIdx.x == 0) {
        float T = time_start;
        for (int k = 0; k < steps; ++k) {
            S->sched[k].t0 = T;
            T = T + h;
        }
        S->counters[0] = 0ull;   // the counters keep the previous call's values: clear them
        S->counters[1] = 0ull;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < steps; k += blockDim.x) {
        StepEntry E{};
        const float T = S->sched[k].t0;
        E.t0 = (T - time_back) / (time_front - time_back);
        E.t1 = ((T + 0.5f * h) - time_back) / (time_front - time_back);
        E.t2 = ((T + h) - time_back) / (time_front - time_back);
        E.slot_back = 0;
        E.slot_front = 1;
        S->sched[k] = E;
    }
}

// The plain step loop of advance_kernel (granite_kernels.cuh) with the same arithmetic:
// no curvature, volumes, expressions, uplift, constants, topography or length abort.
template <int DIM, bool RK4>
__global__ void __launch_bounds__(256) advance_plain_kernel(const __grid_constant__ KParams P,
                                                            NoAllocScratch *S) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < P.n;
    bool alive = valid && P.status[i] == 0;
    const bool was_alive = alive;
    int32_t st = 0;
    V3 p{0.f, 0.f, 0.f};
    if (valid) {
        p.x = P.px[i];
        p.y = P.py[i];
        if (DIM == 3) p.z = P.pz[i];
    }
    unsigned my_steps = 0;
    const int sph = P.sphere && DIM == 2;
    const void *wb = P.wind;
    const void *wf = reinterpret_cast<const char *>(P.wind) + P.wind_stride;
    for (int s = P.s0; s < P.s1 && alive; ++s) {
        const StepEntry E = S->sched[s];
        ++my_steps;
        V3 v;
        if (RK4) {
            const V3 k1c = wind_at<DIM, float>(P, p, E.t0, wb, wf);
            const V3 k1 = sph ? sphere_(P, p.y, k1c) : k1c;
            V3 a{__fmaf_rn(k1.x, P.hh, p.x), __fmaf_rn(k1.y, P.hh, p.y), DIM == 3 ? __fmaf_rn(k1.z, P.hh, p.z) : 0.f};
            const V3 k2c = wind_at<DIM, float>(P, a, E.t1, wb, wf);
            const V3 k2 = sph ? sphere_(P, a.y, k2c) : k2c;
            a = V3{__fmaf_rn(k2.x, P.hh, p.x), __fmaf_rn(k2.y, P.hh, p.y), DIM == 3 ? __fmaf_rn(k2.z, P.hh, p.z) : 0.f};
            const V3 k3c = wind_at<DIM, float>(P, a, E.t1, wb, wf);
            const V3 k3 = sph ? sphere_(P, a.y, k3c) : k3c;
            a = V3{__fmaf_rn(k3.x, P.h, p.x), __fmaf_rn(k3.y, P.h, p.y), DIM == 3 ? __fmaf_rn(k3.z, P.h, p.z) : 0.f};
            const V3 k4c = wind_at<DIM, float>(P, a, E.t2, wb, wf);
            const V3 k4 = sph ? sphere_(P, a.y, k4c) : k4c;
            v.x = (((k1.x + 2.f * k2.x) + 2.f * k3.x) + k4.x) * P.sixth;
            v.y = (((k1.y + 2.f * k2.y) + 2.f * k3.y) + k4.y) * P.sixth;
            v.z = DIM == 3 ? (((k1.z + 2.f * k2.z) + 2.f * k3.z) + k4.z) * P.sixth : 0.f;
        } else {
            const V3 vc = wind_at<DIM, float>(P, p, E.t0, wb, wf);
            v = sph ? sphere_(P, p.y, vc) : vc;
        }
        V3 dp{v.x * P.h, v.y * P.h, DIM == 3 ? v.z * P.h : 0.f};
        if (P.reverse) { dp.x = -dp.x; dp.y = -dp.y; dp.z = -dp.z; }
        V3 np;
        np.x = P.reverse ? p.x - dp.x : p.x + dp.x;
        np.y = P.reverse ? p.y - dp.y : p.y + dp.y;
        np.z = DIM == 3 ? (P.reverse ? p.z - dp.z : p.z + dp.z) : 0.f;
        int32_t abort = 0;
        const float dp2 = dot3(dp, dp, DIM);
        const int bm = DIM == 3 ? 0 : P.border_mode;
        if (bm == 0) {
            if (dp2 < 1e-9f) abort = 4;
            else {
                bool out = np.x - P.off[0] > P.dom[0] || np.x - P.off[0] < 0.f ||
                           np.y - P.off[1] > P.dom[1] || np.y - P.off[1] < 0.f;
                if (DIM == 3) out = out || np.z - P.off[2] > P.dom[2] || np.z - P.off[2] < 0.f;
                if (out) abort = 2;
            }
        } else if (dp2 < 1e-9f) {
            abort = 4;
        } else {
            const float ox = P.off[0], oy = P.off[1], DX = P.dom[0], DY = P.dom[1];
            if (bm == 1) {
                np.x = fmodf(np.x - ox + DX, DX) + ox;
                if (np.y - oy > DY || np.y - oy < 0.f) abort = 2;
            } else if (bm == 2) {
                if (sph) {
                    if (np.x - ox > DX || np.x - ox < 0.f || np.y - oy > DY || np.y - oy < 0.f) abort = 2;
                } else {
                    np.y = fmodf(np.y - oy + DY, DY) + oy;
                    if (np.x - ox > DX || np.x - ox < 0.f) abort = 2;
                }
            } else {
                if (sph) {
                    const float nx_ = np.x - ox, ny_ = np.y - oy, px_ = p.x - ox, py_ = p.y - oy;
                    if (ny_ < 0.f) {
                        const float tx = (-py_) / (ny_ - py_) * (nx_ - px_) + px_;
                        np.y = -ny_ + oy;
                        np.x = fmodf(DX + 180.0f - nx_ + 2.f * tx, DX) + ox;
                    } else if (ny_ >= DY) {
                        const float tx = (DY - py_) / (ny_ - py_) * (nx_ - px_) + px_;
                        np.y = (ny_ - DY) + oy;
                        np.x = fmodf(DX + 180.0f - nx_ + 2.f * tx, DX) + ox;
                    }
                } else {
                    np.y = fmodf(np.y - oy + DY, DY) + oy;
                }
                np.x = fmodf(np.x - ox + DX, DX) + ox;
            }
        }
        st = abort;
        if (abort != 0) alive = false;
        else p = np;
    }
    if (valid && was_alive) {
        P.status[i] = st;
        P.px[i] = p.x;
        P.py[i] = p.y;
        if (DIM == 3) P.pz[i] = p.z;
    }
    const unsigned warp_steps = __reduce_add_sync(0xffffffffu, my_steps);
    const unsigned alive_mask = __ballot_sync(0xffffffffu, valid && alive);
    if ((threadIdx.x & 31) == 0) {
        if (warp_steps) atomicAdd(&S->counters[0], (unsigned long long)warp_steps);
        if (alive_mask) atomicAdd(&S->counters[1], (unsigned long long)__popc(alive_mask));
    }
}

}  // namespace

extern "C" int gr_advance_noalloc(const gr_settings *s, int64_t nz, int64_t ny, int64_t nx, const void *wind_back,
                                  const void *wind_front, float time_back, float time_front, float time_start,
                                  int32_t steps, float *px, float *py, float *pz, int32_t *status, int64_t n,
                                  void *stream, int64_t *particle_steps) {
    if (!s || !wind_back || !wind_front || !px || !py || !status) return err(GR_ERR_USER, "ERROR < USER INPUT | null argument >");
    const int dim = s->space == 0 ? 3 : 2;
    if (dim == 3 && !pz) return err(GR_ERR_USER, "ERROR < USER INPUT | null argument >");
    if (steps < 0 || steps > GR_NOALLOC_MAX_STEPS)
        return err(GR_ERR_USER, "ERROR < USER INPUT | steps must be between 0 and GR_NOALLOC_MAX_STEPS (4096) >");
    if (n < 0 || n > 0x7fffffffLL) return err(GR_ERR_USER, "ERROR < USER INPUT | invalid particle count >");
    if (s->curvature_mode != 0 || s->volume_mode != 0 || s->constants_mode != 0 || (dim == 3 && s->uplift_mode != 0) ||
        s->abort_mode != 0 || s->storage != GR_STORE_F32 || s->compensated || s->windfield_mode != 1 ||
        s->time_mode != 0 || s->minimum_alive > 0)
        return err(GR_ERR_USER, "ERROR < USER INPUT | the allocation-free entry point runs the plain integrator only "
                                "(dynamic wind, float32 storage and time weights; no curvature, volumes, constants, "
                                "uplift, length abort or MinimumAliveParticles) >");
    if (!(s->delta_t > 0.f) || !(time_front > time_back))
        return err(GR_ERR_USER, "ERROR < USER INPUT | DeltaT must be positive and time_front > time_back >");
    if (!(time_start >= time_back) || !(time_start < time_front))
        return err(GR_ERR_USER, "ERROR < USER INPUT | time_start must lie in [time_back, time_front) >");
    if (nx < 1 || ny < 1 || (dim == 3 && nz < 1) || nx * ny * (dim == 3 ? nz : 1) > 0x7fffffffLL)
        return err(GR_ERR_USER, "ERROR < USER INPUT | invalid grid >");
    if (s->device < 0 || s->device >= MAX_DEVICES) return err(GR_ERR_USER, "ERROR < USER INPUT | invalid device >");

    std::lock_guard<std::mutex> lock(g_mutex);
    if (cudaSetDevice(s->device) != cudaSuccess) return err(GR_ERR_RUNTIME, "ERROR < RUNTIME | cudaSetDevice failed >");
    // once per device, with that device current: the device address of the scratch array
    if (!g_scratch_ptr[s->device]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_scratch);
        if (e != cudaSuccess || !ptr) return err(GR_ERR_RUNTIME, "ERROR < RUNTIME | cudaGetSymbolAddress failed >");
        g_scratch_ptr[s->device] = static_cast<NoAllocScratch *>(ptr);
    }
    NoAllocScratch *S = g_scratch_ptr[s->device];
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // the step schedule and cleared counters, built on the device in stream order
    noalloc_schedule_kernel<<<1, 256, 0, st>>>(S, time_back, time_front, time_start, s->delta_t, steps);
    if (cudaGetLastError() != cudaSuccess) return err(GR_ERR_RUNTIME, "ERROR < RUNTIME | schedule launch failed >");
    const float h = s->delta_t;

    KParams P;
    std::memset(&P, 0, sizeof P);
    float scale[3];
    if (s->grid_scale_len == 1) { scale[0] = scale[1] = scale[2] = s->grid_scale[0]; }
    else if (s->grid_scale_len == 2) { scale[0] = s->grid_scale[0]; scale[1] = s->grid_scale[1]; scale[2] = s->grid_scale[0]; }
    else if (s->grid_scale_len == 3) { scale[0] = s->grid_scale[0]; scale[1] = s->grid_scale[1]; scale[2] = s->grid_scale[2]; }
    else return err(GR_ERR_USER, "ERROR < USER INPUT | Invalid GridScale dimension. >");
    float off[3];
    if (s->offset_len == 1) { off[0] = off[1] = off[2] = s->offset[0]; }
    else if (s->grid_scale_len == 2 && s->offset_len >= 2) { off[0] = s->offset[0]; off[1] = s->offset[1]; off[2] = s->offset[0]; }
    else if (s->grid_scale_len == 3 && s->offset_len >= 3) { off[0] = s->offset[0]; off[1] = s->offset[1]; off[2] = s->offset[2]; }
    else return err(GR_ERR_USER, "ERROR < USER INPUT | Invalid Offset dimension. >");
    const float g[3] = {(float)nx, (float)ny, (float)(dim == 3 ? nz : 0)};
    for (int d = 0; d < 3; ++d) {
        P.scale[d] = scale[d];
        P.inv_scale[d] = 1.0f / scale[d];
        P.off[d] = off[d];
        P.dom[d] = g[d] * scale[d];
    }
    P.nx = (int32_t)nx; P.ny = (int32_t)ny; P.nz = (int32_t)(dim == 3 ? nz : 1); P.dim = dim;
    P.fn[0] = (float)P.nx; P.fn[1] = (float)P.ny; P.fn[2] = (float)P.nz;
    P.wind = wind_back;
    P.wind_stride = reinterpret_cast<const char *>(wind_front) - reinterpret_cast<const char *>(wind_back);
    P.px = px; P.py = py; P.pz = pz; P.status = status;
    P.n = n;
    P.s0 = 0;
    P.s1 = steps;
    P.h = h;
    P.hh = 0.5f * h;
    P.sixth = 1.0f / 6;
    P.inv_2h = 1.0f / (2.0f * h);
    P.inv_hh = 1.0f / (h * h);
    P.sphere_radius = s->sphere_radius;
    P.filter_weights = s->filter_weights ? 1 : 0;
    P.wind_dynamic = 1;
    P.dyn_any = 1;
    P.border_mode = dim == 2 ? s->border_mode : 0;
    P.reverse = s->reverse ? 1 : 0;
    P.sphere = dim == 2 && s->sphere_radius > 0.f;
    const int threads = 256;
    const unsigned blocks = (unsigned)std::max<int64_t>(1, (n + threads - 1) / threads);
    const bool rk4 = s->integrator == 1;
    if (dim == 3) {
        if (rk4) advance_plain_kernel<3, true><<<blocks, threads, 0, st>>>(P, S);
        else advance_plain_kernel<3, false><<<blocks, threads, 0, st>>>(P, S);
    } else {
        if (rk4) advance_plain_kernel<2, true><<<blocks, threads, 0, st>>>(P, S);
        else advance_plain_kernel<2, false><<<blocks, threads, 0, st>>>(P, S);
    }
    if (cudaGetLastError() != cudaSuccess) return err(GR_ERR_RUNTIME, "ERROR < RUNTIME | launch failed >");
    if (particle_steps) {
        unsigned long long c = 0;
        if (cudaMemcpyAsync(&c, &S->counters[0], sizeof c, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return err(GR_ERR_RUNTIME, "ERROR < RUNTIME | reading the step counter failed >");
        *particle_steps = (int64_t)c;
    }
    return GR_OK;
}
