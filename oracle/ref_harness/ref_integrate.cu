// ref_integrate.cu — runs the reference's own `integrate` kernel (TEST INFRASTRUCTURE ONLY).
//
// Compiled from the reference's sources where they lie (-I <reference>/source) by
// oracle/ref_harness/Makefile into oracle/_ref/libref_integrate.so.  The kernel template
// (source/granite/TrajectoryIntegrator.tpp:108-457 with TrajectoryIntegrator.icc) is the
// reference's code, instantiated unmodified; everything in this file is a restatement of the
// host side it needs, because the reference's TrajectoryIntegrator.cpp depends on the
// un-vendored cpp-peglib:
//  * textures exactly as loadTexture3D / loadTexture2D set them up (cpp:444-583): 3D
//    cudaArray, border addressing, linear filtering; 2D pitch-linear, default addressing;
//  * SimulationData as compute_ fills it (tpp:515-712);
//  * the step loop of computeLoop_ / computeLoopGPU_ (tpp:778-995), including its launch
//    shape THREADS = min(maxThreadsPerBlock, N) / 2, BLOCKS = min(sdiv(THREADS, N), ...)
//    (tpp:790-796) when blocks_fixed == 0, and the synchronous copy of every saved step.
// Only tests/ (golden fixtures) use it, on the GPU.
#include "granite/TrajectoryIntegrator.hpp"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

using namespace granite;
using my::math::Vec2;
using my::math::Vec3;

// 2D Euler, Block, no curvature / volumes / expressions (the double-gyre configuration)
#define REF_ARGS_2D Vec2, Space::Space2D, Integrator::ExplicitEuler, BorderMode::Block, CurvatureMode::Off,  \
    AbortMode::Time, UpLiftMode::Off, WindfieldMode::Dynamic, ConstantsMode::Off, AdditionalVolumeMode::Off, \
    false, false, false, false, false
// 3D RK4, TotalCurvature, one constant volume, expressions (the Fourier-field configuration)
#define REF_ARGS_3D Vec3, Space::Space3D, Integrator::ClassicRungeKutta, BorderMode::Block,                  \
    CurvatureMode::TotalCurvature, AbortMode::Time, UpLiftMode::Off, WindfieldMode::Dynamic,                  \
    ConstantsMode::Off, AdditionalVolumeMode::Constant, false, false, false, true, true
// 3D RK4 plain
#define REF_ARGS_3P Vec3, Space::Space3D, Integrator::ClassicRungeKutta, BorderMode::Block, CurvatureMode::Off, \
    AbortMode::Time, UpLiftMode::Off, WindfieldMode::Dynamic, ConstantsMode::Off, AdditionalVolumeMode::Off,   \
    false, false, false, false, false
// 3D Euler plain (one step of it samples the texture filter directly)
#define REF_ARGS_3E Vec3, Space::Space3D, Integrator::ExplicitEuler, BorderMode::Block, CurvatureMode::Off,    \
    AbortMode::Time, UpLiftMode::Off, WindfieldMode::Dynamic, ConstantsMode::Off, AdditionalVolumeMode::Off,   \
    false, false, false, false, false

extern "C" {

typedef struct {
    int32_t variant;          // 0: 2D Euler plain, 1: 3D RK4 curvature+volume+expression, 2: 3D RK4 plain,
                              // 3: 3D Euler plain
    int32_t blocks_fixed;     // 0: launch shape as shipped; 1: BLOCKS = ceil(N / THREADS)
    float delta_t, data_time_distance, maximum_simulation_time;
    int64_t save_interval;
    float scale[3], offset[3];
    int64_t nx, ny, nz;
    int32_t n_snapshots;
    const float *const *wind;     // [snapshot * dim] planes
    const float *volume;          // constant volume (variant 1)
    const ASTANode *ast;          // flat pre-order AST (variant 1)
    int32_t ast_len;
    int64_t n;
    const float *seeds;           // n * dim
    int64_t step_limit;           // < 0: none
    // outputs
    int64_t max_records;
    float *positions;             // [max_records][n][dim]
    int32_t *status;              // [n]
    float *total_curvature;       // [n]
    float *volume_info;           // [max_records][n]
    float *compute_info;          // [max_records][n]
    int64_t records, info_records, steps, windows;
    double loop_ms;               // wall time of the step loop
    int32_t threads, blocks;
    char message[256];
    int32_t count_steps;          // 1: count the particle-steps (alive particles at each launch)
    int64_t particle_steps;       // counted when count_steps
    int64_t h2d_bytes, d2h_bytes; // copies made inside the step loop
} ref_args;

}  // extern "C"

namespace {

#define RCK(x)                                                                                      \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) {                                                                    \
            snprintf(a->message, sizeof a->message, "%s (line %d)", cudaGetErrorString(e_), __LINE__); \
            return 1;                                                                               \
        }                                                                                           \
    } while (0)

// Particles alive (status Time) before a launch, summed into *out: the particle-steps of that
// launch.  The harness's own bookkeeping, not part of the reference.
__global__ void count_alive_kernel(const AbortReason *status, int64_t n, unsigned long long *out) {
    unsigned c = 0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        c += status[i] == AbortReason::Time ? 1u : 0u;
    c = __reduce_add_sync(0xffffffffu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, (unsigned long long)c);
}

struct Tex {
    cudaTextureObject_t obj = 0;
    cudaArray_t arr = nullptr;
    float *lin = nullptr;
    size_t pitch = 0;
};

// loadTexture3D (cpp:444-514)
int load3(ref_args *a, Tex &t, const float *host) {
    const cudaExtent ext = make_cudaExtent(a->nx, a->ny, a->nz);
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    if (!t.arr) RCK(cudaMalloc3DArray(&t.arr, &cd, ext));
    cudaMemcpy3DParms p;
    memset(&p, 0, sizeof p);
    p.srcPtr = make_cudaPitchedPtr(const_cast<float *>(host), ext.width * sizeof(float), ext.width, ext.height);
    p.dstArray = t.arr;
    p.extent = ext;
    p.kind = cudaMemcpyHostToDevice;
    RCK(cudaMemcpy3D(&p));
    if (!t.obj) {
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof rd);
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = t.arr;
        cudaTextureDesc td;
        memset(&td, 0, sizeof td);
        td.normalizedCoords = false;
        td.filterMode = cudaFilterModeLinear;
        for (int i = 0; i < 3; ++i) td.addressMode[i] = cudaAddressModeBorder;
        td.readMode = cudaReadModeElementType;
        RCK(cudaCreateTextureObject(&t.obj, &rd, &td, nullptr));
    }
    return 0;
}

// loadTexture2D (cpp:516-583)
int load2(ref_args *a, Tex &t, const float *host) {
    if (!t.lin) RCK(cudaMallocPitch(&t.lin, &t.pitch, sizeof(float) * a->nx, a->ny));
    RCK(cudaMemcpy2D(t.lin, t.pitch, host, sizeof(float) * a->nx, sizeof(float) * a->nx, a->ny,
                     cudaMemcpyHostToDevice));
    if (!t.obj) {
        cudaResourceDesc rd;
        memset(&rd, 0, sizeof rd);
        rd.resType = cudaResourceTypePitch2D;
        rd.res.pitch2D.devPtr = t.lin;
        rd.res.pitch2D.pitchInBytes = t.pitch;
        rd.res.pitch2D.width = a->nx;
        rd.res.pitch2D.height = a->ny;
        rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
        cudaTextureDesc td;
        memset(&td, 0, sizeof td);
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = false;
        td.filterMode = cudaFilterModeLinear;
        RCK(cudaCreateTextureObject(&t.obj, &rd, &td, nullptr));
    }
    return 0;
}

void free_tex(Tex &t) {
    if (t.obj) cudaDestroyTextureObject(t.obj);
    if (t.arr) cudaFreeArray(t.arr);
    if (t.lin) cudaFree(t.lin);
}

template <typename VEC_T>
void launch(int variant, int blocks, int threads, const SimulationData<VEC_T> &d);

template <>
void launch<Vec2>(int, int blocks, int threads, const SimulationData<Vec2> &d) {
    integrate<REF_ARGS_2D><<<blocks, threads>>>(d);
}

template <>
void launch<Vec3>(int variant, int blocks, int threads, const SimulationData<Vec3> &d) {
    if (variant == 1) integrate<REF_ARGS_3D><<<blocks, threads>>>(d);
    else if (variant == 3) integrate<REF_ARGS_3E><<<blocks, threads>>>(d);
    else integrate<REF_ARGS_3P><<<blocks, threads>>>(d);
}

template <typename VEC_T>
int run(ref_args *a) {
    constexpr int DIM = sizeof(VEC_T) / sizeof(float);
    const int64_t n = a->n;
    const bool extras = a->variant == 1;
    Tex wind[3][3];   // [slot][component]
    Tex vol;
    int back = 0, front = 1, cache = 2;
    a->h2d_bytes = a->d2h_bytes = 0;
    a->particle_steps = 0;
    const int64_t plane_bytes = a->nx * a->ny * (DIM == 3 ? a->nz : 1) * (int64_t)sizeof(float);
    auto load_snapshot = [&](int slot, int s) -> int {
        for (int c = 0; c < DIM; ++c) {
            const float *h = a->wind[(int64_t)s * DIM + c];
            if ((DIM == 3 ? load3(a, wind[slot][c], h) : load2(a, wind[slot][c], h))) return 1;
        }
        a->h2d_bytes += DIM * plane_bytes;
        return 0;
    };
    // initializeData (cpp:146-259): snapshot 0, the constant volume, then one loader step
    if (load_snapshot(0, 0)) return 1;
    if (extras && load3(a, vol, a->volume)) return 1;
    if (a->n_snapshots < 2) {
        snprintf(a->message, sizeof a->message, "Cannot increment loader.");
        return 1;
    }
    if (load_snapshot(1, 1)) return 1;
    int loaded = 2;

    // compute_ (tpp:467-712)
    VEC_T *buf[2] = {nullptr, nullptr};
    RCK(cudaMalloc(&buf[0], n * sizeof(VEC_T)));
    RCK(cudaMalloc(&buf[1], n * sizeof(VEC_T)));
    RCK(cudaMemcpy(buf[0], a->seeds, n * sizeof(VEC_T), cudaMemcpyHostToDevice));
    int swap_index = 0;   // SwapChain: front = buf[index], back = buf[1 - index]
    AbortReason *status = nullptr;
    RCK(cudaMalloc(&status, n * sizeof(AbortReason)));
    RCK(cudaMemset(status, 0, n * sizeof(AbortReason)));
    SimulationData<VEC_T> d;
    d.Status = status;
    d.NumParticles = n;
    d.Radius = 0.f;
    d.GridScale.X = a->scale[0]; d.GridScale.Y = a->scale[1]; d.GridScale.Z = a->scale[2];
    d.Domain.X = a->nx * a->scale[0]; d.Domain.Y = a->ny * a->scale[1]; d.Domain.Z = a->nz * a->scale[2];
    d.Offset.X = a->offset[0]; d.Offset.Y = a->offset[1]; d.Offset.Z = a->offset[2];
    float *tc = nullptr, *vinfo = nullptr, *cinfo = nullptr;
    ASTANode *ast = nullptr;
    if (extras) {
        RCK(cudaMalloc(&tc, n * sizeof(float)));
        RCK(cudaMemset(tc, 0, n * sizeof(float)));
        d.TotalCurvature = tc;
        d.NumAdditionalVolumes = 1;
        RCK(cudaMalloc(&vinfo, n * sizeof(float)));
        RCK(cudaMemset(vinfo, 0, n * sizeof(float)));   // the reference leaves it uninitialised
        d.ParticleVolumeInfo[0] = vinfo;
        d.NumAdditionalCompute = 1;
        RCK(cudaMalloc(&ast, sizeof(ASTANode) * a->ast_len));
        RCK(cudaMemcpy(ast, a->ast, sizeof(ASTANode) * a->ast_len, cudaMemcpyHostToDevice));
        d.ASTNodes[0] = ast;
        d.ASTSizes[0] = a->ast_len;
        RCK(cudaMalloc(&cinfo, n * sizeof(float)));
        RCK(cudaMemset(cinfo, 0, n * sizeof(float)));
        d.ParticleComputeInfo[0] = cinfo;
        d.AdditionalVolumesBack[0] = vol.obj;
    }
    d.NumAdditionalConstants = 0;
    d.DeltaT = a->delta_t;

    // launch shape (tpp:787-796)
    cudaDeviceProp prop;
    RCK(cudaGetDeviceProperties(&prop, 0));
    const unsigned threads = (unsigned)(std::min((size_t)prop.maxThreadsPerBlock, (size_t)n)) / 2;
    unsigned blocks = (unsigned)std::min<size_t>((threads + n - 1) / n, (size_t)prop.maxThreadsDim[0]);
    if (a->blocks_fixed) blocks = (unsigned)((n + threads - 1) / threads);
    a->threads = (int32_t)threads;
    a->blocks = (int32_t)blocks;

    std::vector<VEC_T> host_pos(n);
    std::vector<float> host_f(n);
    a->records = 0;
    a->info_records = 0;
    auto save = [&](bool time_positive) -> int {
        (void)time_positive;
        VEC_T *f = buf[swap_index];
        if (a->records < a->max_records) {
            RCK(cudaMemcpy(a->positions + a->records * n * DIM, f, n * sizeof(VEC_T), cudaMemcpyDeviceToHost));
            a->d2h_bytes += n * sizeof(VEC_T);
        }
        a->records++;
        if (extras) {
            if (a->info_records < a->max_records) {
                RCK(cudaMemcpy(a->compute_info + a->info_records * n, cinfo, n * sizeof(float), cudaMemcpyDeviceToHost));
                RCK(cudaMemcpy(a->volume_info + a->info_records * n, vinfo, n * sizeof(float), cudaMemcpyDeviceToHost));
                a->d2h_bytes += 2 * n * sizeof(float);
            }
            a->info_records++;
        }
        return 0;
    };
    // record 0 = the seeds
    if (a->max_records > 0) memcpy(a->positions, a->seeds, n * sizeof(VEC_T));
    a->records = 1;

    unsigned long long *steps_dev = nullptr;
    if (a->count_steps) {
        RCK(cudaMalloc(&steps_dev, sizeof(unsigned long long)));
        RCK(cudaMemset(steps_dev, 0, sizeof(unsigned long long)));
    }
    a->h2d_bytes = 0;   // copies before the loop are set-up, not counted

    // computeLoop_ / computeLoopGPU_ (tpp:778-995)
    float time = 0.f, max_wt = a->data_time_distance;
    const float limit = a->maximum_simulation_time / a->delta_t;
    size_t counter = 0, sim = 0;
    a->windows = 0;
    const auto t_start = std::chrono::steady_clock::now();
    for (;;) {
        a->windows++;
        d.TimeBack = counter * a->data_time_distance;
        d.TimeFront = (counter + 1) * a->data_time_distance;
        for (int c = 0; c < DIM; ++c) {
            d.WindfieldBack[c] = wind[back][c].obj;
            d.WindfieldFront[c] = wind[front][c].obj;
        }
        d.Time = time;
        while ((float)sim < limit && (a->step_limit < 0 || (int64_t)sim < a->step_limit)) {
            swap_index = (swap_index + 1) % 2;
            d.FrontParticles = buf[swap_index];
            d.BackParticles = buf[(swap_index + 1) % 2];
            if (steps_dev) count_alive_kernel<<<148 * 4, 256>>>(status, (int64_t)n, steps_dev);
            launch<VEC_T>(a->variant, blocks, threads, d);
            RCK(cudaDeviceSynchronize());
            RCK(cudaGetLastError());
            if (a->save_interval != 0 && sim % a->save_interval == 0)
                if (save(d.Time > 0)) return 1;
            d.Time += d.DeltaT;
            ++sim;
            if (d.Time >= max_wt) break;
        }
        time = d.Time;
        if (loaded < a->n_snapshots) {
            if (load_snapshot(cache, loaded)) return 1;
            ++loaded;
            max_wt += a->data_time_distance;
            const int tmp = back;
            back = front;
            front = cache;
            cache = tmp;
            ++counter;
        } else {
            break;
        }
        if (!((float)sim < limit) || (a->step_limit >= 0 && (int64_t)sim >= a->step_limit)) break;
    }
    if (a->save_interval == 0)
        if (save(d.Time > 0)) return 1;
    a->loop_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    a->steps = (int64_t)sim;
    if (steps_dev) {
        unsigned long long c = 0;
        RCK(cudaMemcpy(&c, steps_dev, sizeof c, cudaMemcpyDeviceToHost));
        a->particle_steps = (int64_t)c;
        cudaFree(steps_dev);
    }
    RCK(cudaMemcpy(a->status, status, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (extras && a->total_curvature) RCK(cudaMemcpy(a->total_curvature, tc, n * sizeof(float), cudaMemcpyDeviceToHost));

    cudaFree(buf[0]);
    cudaFree(buf[1]);
    cudaFree(status);
    if (tc) cudaFree(tc);
    if (vinfo) cudaFree(vinfo);
    if (cinfo) cudaFree(cinfo);
    if (ast) cudaFree(ast);
    for (auto &s : wind)
        for (auto &t : s) free_tex(t);
    free_tex(vol);
    return 0;
}

}  // namespace

extern "C" int ref_run(ref_args *a) {
    a->message[0] = 0;
    if (a->n < 2) {
        snprintf(a->message, sizeof a->message, "the reference's launch shape needs at least 2 particles");
        return 1;
    }
    return a->variant == 0 ? run<Vec2>(a) : run<Vec3>(a);
}
