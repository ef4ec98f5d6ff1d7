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
template <typename A>
int load3(A *a, Tex &t, const float *host) {
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
template <typename A>
int load2(A *a, Tex &t, const float *host) {
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

// ------------------------------------------------------------------------------------------
// The option matrix: further instantiations of the reference's kernel, each with the data its
// options read (textures, per-particle arrays) set up as compute_ / computeLoop_ /
// computeLoopGPU_ / initializeData / updateData do (tpp:467-995, cpp:146-360, 635-660).
// Harness-side deviations, where the reference's host code is defective: dynamic constants are
// stored by their constant index (updateData indexes them from Reference_F0, cpp:319-320, past
// the end of its arrays).  Dynamic volumes are not instantiated: the kernel samples the wind's
// u component for them (icc:52-68).

#define OPT_VARIANTS(X)                                                                                                \
    X(10, Vec2, Space2D, ExplicitEuler, LoopX, Off, Time, Off, Dynamic, Off, Off, false, false, false, false)           \
    X(11, Vec2, Space2D, ClassicRungeKutta, LoopY, Off, Time, Off, Dynamic, Off, Off, false, false, false, false)       \
    X(12, Vec2, Space2D, ClassicRungeKutta, LoopXY, Off, Time, Off, Dynamic, Off, Off, false, false, false, false)      \
    X(13, Vec2, Space2D, ClassicRungeKutta, LoopXY, Off, Time, Off, Dynamic, Off, Off, false, false, true, false)       \
    X(14, Vec2, Space2D, ExplicitEuler, LoopY, Off, Time, Off, Dynamic, Off, Off, false, false, true, false)            \
    X(15, Vec2, Space2D, ClassicRungeKutta, Block, FastTotalCurvature, Time, Off, Dynamic, Off, Off, false, true, false, \
      false)                                                                                                            \
    X(16, Vec2, Space2D, ClassicRungeKutta, Block, Off, Time, Off, Constant, Off, Off, false, false, false, false)      \
    X(17, Vec2, Space2D, ClassicRungeKutta, LoopX, FastTotalCurvature, Time, Off, Dynamic, Off, Off, false, false, true,\
      false)                                                                                                            \
    X(20, Vec3, Space3D, ClassicRungeKutta, Block, IndividualAndTotalCurvature, Length, Off, Dynamic, Off, Off, false,  \
      false, false, false)                                                                                              \
    X(21, Vec3, Space3D, ExplicitEuler, Block, Off, FitLength, Constant, Dynamic, Off, Off, false, false, false, false) \
    X(22, Vec3, Space3D, ClassicRungeKutta, Block, Off, Time, Dynamic, Dynamic, Off, Off, true, false, false, false)    \
    X(23, Vec3, Space3D, ClassicRungeKutta, Block, TotalCurvature, Time, Off, Dynamic, Constant, Constant, false, false,\
      false, true)                                                                                                      \
    X(24, Vec3, Space3D, ClassicRungeKutta, Block, Off, Time, Off, Dynamic, Dynamic, Off, false, true, false, true)     \
    X(25, Vec3, Space3D, ExplicitEuler, Block, TotalCurvature, Length, Off, Constant, Off, Off, false, true, false, false)

extern "C" {

typedef struct {
    // the variant: enum values of the reference's IntegratorSettings (IntegratorSettings.hpp:16-74)
    int32_t dim, integrator, border_mode, curvature_mode, abort_mode, uplift_mode, windfield_mode, constants_mode,
        volume_mode, use_topography, reverse, use_sphere, comp_additional;
    int32_t blocks_fixed;
    float delta_t, data_time_distance, maximum_simulation_time, maximum_length, sphere_radius;
    int64_t save_interval;
    float scale[3], offset[3];
    int64_t nx, ny, nz;
    int32_t n_snapshots;
    const float *const *wind;        // [snapshot * dim] planes
    int32_t n_volumes;               // 0 or 1 (constant volume)
    const float *const *volumes;     // [n_volumes] planes
    int32_t n_constants;             // 0..4
    const float *const *constants;   // [snapshot * n_constants] arrays of n (snapshot 0 only if constant)
    const float *const *uplift;      // [snapshot] arrays of n * dim (snapshot 0 only if constant)
    const float *topography;         // (ny, nx) or null
    const ASTANode *ast;             // one flat expression (comp_additional)
    int32_t ast_len;
    int64_t n;
    const float *seeds;
    // outputs
    int64_t max_records;
    float *positions;                // [max_records][n][dim]
    int32_t *status;
    float *total_curvature, *lengths;
    float *curvature;                // [max_records][n]
    float *volume_info;              // [max_records][n]
    float *compute_info;             // [max_records][n]
    int64_t records, curvature_records, info_records, steps, windows;
    char message[256];
} ref_opt_args;

}  // extern "C"

namespace {

template <typename VEC_T>
using OptLaunch = void (*)(int blocks, int threads, const SimulationData<VEC_T> &d);

struct OptEntry {
    int id, dim, integrator, border, curvature, abort_mode, uplift, windfield, constants, volume, topo, reverse, sphere,
        comp;
    void *fn;
};

#define OPT_KERNEL(ID, VT, SP, IN, BM, CM, AM, UM, WM, KM, VM, TOPO, REV, SPH, COMP)                                   \
    void opt_launch_##ID(int blocks, int threads, const SimulationData<VT> &d) {                                       \
        integrate<VT, Space::SP, Integrator::IN, BorderMode::BM, CurvatureMode::CM, AbortMode::AM, UpLiftMode::UM,      \
                  WindfieldMode::WM, ConstantsMode::KM, AdditionalVolumeMode::VM, TOPO, REV, SPH, COMP,                 \
                  AdditionalVolumeMode::VM != AdditionalVolumeMode::Off><<<blocks, threads>>>(d);                       \
    }
OPT_VARIANTS(OPT_KERNEL)
#undef OPT_KERNEL

#define OPT_ENTRY(ID, VT, SP, IN, BM, CM, AM, UM, WM, KM, VM, TOPO, REV, SPH, COMP)                                    \
    {ID, (int)sizeof(VT) / (int)sizeof(float), (int)Integrator::IN, (int)BorderMode::BM, (int)CurvatureMode::CM,        \
     (int)AbortMode::AM, (int)UpLiftMode::UM, (int)WindfieldMode::WM, (int)ConstantsMode::KM,                           \
     (int)AdditionalVolumeMode::VM, TOPO, REV, SPH, COMP, (void *)&opt_launch_##ID},
const OptEntry kOpt[] = {OPT_VARIANTS(OPT_ENTRY)};
#undef OPT_ENTRY

template <typename VEC_T>
int run_opt(ref_opt_args *a, OptLaunch<VEC_T> fn) {
    constexpr int DIM = sizeof(VEC_T) / sizeof(float);
    const int64_t n = a->n;
    const bool dyn_wind = a->windfield_mode == 1;
    const bool dyn_any = dyn_wind || a->uplift_mode == 2 || a->volume_mode == 2 || a->constants_mode == 2;
    Tex wind[3][3], vol, topo;
    float *cons[3][4] = {};
    VEC_T *lift[3] = {};
    int back = 0, front = 1, cache = 2;
    // updateData(index) of the snapshot s (cpp:262-360), and its first call in initializeData
    auto load_snapshot = [&](int slot, int s, bool first) -> int {
        if (first || dyn_wind)
            for (int c = 0; c < DIM; ++c) {
                const float *h = a->wind[(int64_t)s * DIM + c];
                if ((DIM == 3 ? load3(a, wind[slot][c], h) : load2(a, wind[slot][c], h))) return 1;
            }
        if (a->constants_mode != 0 && (first || a->constants_mode == 2))
            for (int k = 0; k < a->n_constants; ++k) {
                if (!cons[slot][k]) RCK(cudaMalloc(&cons[slot][k], n * sizeof(float)));
                RCK(cudaMemcpy(cons[slot][k], a->constants[(int64_t)s * a->n_constants + k], n * sizeof(float),
                               cudaMemcpyHostToDevice));
            }
        if (a->uplift_mode != 0 && (first || a->uplift_mode == 2)) {
            if (!lift[slot]) RCK(cudaMalloc(&lift[slot], n * sizeof(VEC_T)));
            RCK(cudaMemcpy(lift[slot], a->uplift[s], n * sizeof(VEC_T), cudaMemcpyHostToDevice));
        }
        return 0;
    };
    // initializeData (cpp:146-259)
    if (load_snapshot(0, 0, true)) return 1;
    if (a->volume_mode == 1 && a->n_volumes > 0)
        if ((DIM == 3 ? load3(a, vol, a->volumes[0]) : load2(a, vol, a->volumes[0]))) return 1;
    int loaded = 1;
    if (dyn_any) {
        if (a->n_snapshots < 2) {
            snprintf(a->message, sizeof a->message, "Cannot increment loader.");
            return 1;
        }
        if (load_snapshot(1, 1, false)) return 1;
        loaded = 2;
    }
    // initializeTopography (cpp:635-660): a 2D pitch texture of the (ny, nx) plane
    if (a->use_topography) {
        ref_opt_args t2 = *a;
        t2.nz = 1;
        if (load2(&t2, topo, a->topography)) {
            memcpy(a->message, t2.message, sizeof a->message);
            return 1;
        }
    }

    // compute_ (tpp:467-712)
    VEC_T *buf[2] = {nullptr, nullptr};
    RCK(cudaMalloc(&buf[0], n * sizeof(VEC_T)));
    RCK(cudaMalloc(&buf[1], n * sizeof(VEC_T)));
    RCK(cudaMemcpy(buf[0], a->seeds, n * sizeof(VEC_T), cudaMemcpyHostToDevice));
    int swap_index = 0;
    AbortReason *status = nullptr;
    RCK(cudaMalloc(&status, n * sizeof(AbortReason)));
    RCK(cudaMemset(status, 0, n * sizeof(AbortReason)));
    SimulationData<VEC_T> d;
    d.Status = status;
    d.NumParticles = n;
    d.Radius = a->sphere_radius;
    d.GridScale.X = a->scale[0]; d.GridScale.Y = a->scale[1]; d.GridScale.Z = a->scale[2];
    d.Domain.X = a->nx * a->scale[0]; d.Domain.Y = a->ny * a->scale[1]; d.Domain.Z = a->nz * a->scale[2];
    d.Offset.X = a->offset[0]; d.Offset.Y = a->offset[1]; d.Offset.Z = a->offset[2];
    float *len = nullptr, *curv = nullptr, *tc = nullptr, *vinfo = nullptr, *cinfo = nullptr;
    VEC_T *lastdir = nullptr;
    ASTANode *ast = nullptr;
    if (a->abort_mode != 0) {
        RCK(cudaMalloc(&len, n * sizeof(float)));
        RCK(cudaMemset(len, 0, n * sizeof(float)));
        d.MaximumLength = a->maximum_length;
        d.CurrentLength = len;
    }
    if (a->curvature_mode != 0) {
        if (a->curvature_mode == 3) {
            RCK(cudaMalloc(&curv, n * sizeof(float)));
            RCK(cudaMemset(curv, 0, n * sizeof(float)));
            d.Curvature = curv;
        }
        if (a->curvature_mode == 2) RCK(cudaMalloc(&lastdir, n * sizeof(VEC_T)));
        RCK(cudaMalloc(&tc, n * sizeof(float)));
        RCK(cudaMemset(tc, 0, n * sizeof(float)));
        d.TotalCurvature = tc;
        d.LastDirections = lastdir;
    }
    d.NumAdditionalVolumes = 0;
    if (a->volume_mode != 0) {
        d.NumAdditionalVolumes = a->n_volumes;
        if (a->n_volumes > 0) {
            RCK(cudaMalloc(&vinfo, n * sizeof(float)));
            RCK(cudaMemset(vinfo, 0, n * sizeof(float)));   // the reference leaves it uninitialised
            d.ParticleVolumeInfo[0] = vinfo;
        }
    }
    d.NumAdditionalCompute = 0;
    if (a->comp_additional) {
        d.NumAdditionalCompute = 1;
        RCK(cudaMalloc(&ast, sizeof(ASTANode) * a->ast_len));
        RCK(cudaMemcpy(ast, a->ast, sizeof(ASTANode) * a->ast_len, cudaMemcpyHostToDevice));
        d.ASTNodes[0] = ast;
        d.ASTSizes[0] = a->ast_len;
        RCK(cudaMalloc(&cinfo, n * sizeof(float)));
        RCK(cudaMemset(cinfo, 0, n * sizeof(float)));
        d.ParticleComputeInfo[0] = cinfo;
    }

    // computeLoop_ (tpp:764-918)
    cudaDeviceProp prop;
    RCK(cudaGetDeviceProperties(&prop, 0));
    const unsigned threads = (unsigned)(std::min((size_t)prop.maxThreadsPerBlock, (size_t)n)) / 2;
    unsigned blocks = (unsigned)std::min<size_t>((threads + n - 1) / n, (size_t)prop.maxThreadsDim[0]);
    if (a->blocks_fixed) blocks = (unsigned)((n + threads - 1) / threads);
    if (!dyn_wind)
        for (int c = 0; c < DIM; ++c) d.WindfieldBack[c] = wind[0][c].obj;
    if (a->volume_mode == 1 && a->n_volumes > 0) d.AdditionalVolumesBack[0] = vol.obj;
    if (a->uplift_mode == 1) d.LiftBack = lift[0];
    d.NumAdditionalConstants = a->n_constants;
    if (a->constants_mode == 1)
        for (int k = 0; k < a->n_constants; ++k) {
            d.ComputeDataBack[k] = cons[0][k];
            d.ComputeDataFront[k] = cons[0][k];
        }
    d.DeltaT = a->delta_t;

    std::vector<float> host_f(n);
    a->records = a->curvature_records = a->info_records = 0;
    // copyParticleInfo (tpp:997-1049)
    auto save = [&]() -> int {
        VEC_T *f = buf[swap_index];
        if (a->records < a->max_records)
            RCK(cudaMemcpy(a->positions + a->records * n * DIM, f, n * sizeof(VEC_T), cudaMemcpyDeviceToHost));
        a->records++;
        if (a->curvature_mode == 3 && d.Time > 0) {
            if (a->curvature_records < a->max_records)
                RCK(cudaMemcpy(a->curvature + a->curvature_records * n, curv, n * sizeof(float), cudaMemcpyDeviceToHost));
            a->curvature_records++;
        }
        if (cinfo || vinfo) {
            if (a->info_records < a->max_records) {
                if (cinfo)
                    RCK(cudaMemcpy(a->compute_info + a->info_records * n, cinfo, n * sizeof(float), cudaMemcpyDeviceToHost));
                if (vinfo)
                    RCK(cudaMemcpy(a->volume_info + a->info_records * n, vinfo, n * sizeof(float), cudaMemcpyDeviceToHost));
            }
            a->info_records++;
        }
        return 0;
    };
    if (a->max_records > 0) memcpy(a->positions, a->seeds, n * sizeof(VEC_T));
    a->records = 1;

    size_t counter = 0, sim = 0;
    float max_wt = a->data_time_distance;
    const float limit = a->maximum_simulation_time / a->delta_t;
    d.Time = 0.f;
    a->windows = 0;
    do {
        // computeLoopGPU_ (tpp:920-995)
        a->windows++;
        const float window_end = dyn_any ? max_wt : a->maximum_simulation_time;
        if (a->use_topography) d.Topography = topo.obj;
        d.TimeBack = counter * a->data_time_distance;
        d.TimeFront = (counter + 1) * a->data_time_distance;
        if (dyn_wind)
            for (int c = 0; c < DIM; ++c) {
                d.WindfieldBack[c] = wind[back][c].obj;
                d.WindfieldFront[c] = wind[front][c].obj;
            }
        if (a->uplift_mode == 2) {
            d.LiftBack = lift[back];
            d.LiftFront = lift[front];
        }
        if (a->constants_mode == 2)
            for (int k = 0; k < a->n_constants; ++k) {
                d.ComputeDataBack[k] = cons[back][k];
                d.ComputeDataFront[k] = cons[front][k];
            }
        while ((float)sim < limit) {
            swap_index = (swap_index + 1) % 2;
            d.FrontParticles = buf[swap_index];
            d.BackParticles = buf[(swap_index + 1) % 2];
            fn(blocks, threads, d);
            RCK(cudaDeviceSynchronize());
            RCK(cudaGetLastError());
            if (a->save_interval != 0 && sim % a->save_interval == 0)
                if (save()) return 1;
            d.Time += d.DeltaT;
            ++sim;
            if (d.Time >= window_end) break;
        }
        if (dyn_any) {
            if (loaded < a->n_snapshots) {   // _loader.step() returned true
                if (load_snapshot(cache, loaded, false)) return 1;
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
        }
    } while (dyn_wind && (float)sim < limit);
    if (a->save_interval == 0)
        if (save()) return 1;
    a->steps = (int64_t)sim;
    RCK(cudaMemcpy(a->status, status, n * sizeof(int32_t), cudaMemcpyDeviceToHost));
    if (tc && a->total_curvature) RCK(cudaMemcpy(a->total_curvature, tc, n * sizeof(float), cudaMemcpyDeviceToHost));
    if (len && a->lengths) RCK(cudaMemcpy(a->lengths, len, n * sizeof(float), cudaMemcpyDeviceToHost));

    cudaFree(buf[0]); cudaFree(buf[1]); cudaFree(status);
    for (float *p : {len, curv, tc, vinfo, cinfo}) if (p) cudaFree(p);
    if (lastdir) cudaFree(lastdir);
    if (ast) cudaFree(ast);
    for (auto &sl : cons) for (float *p : sl) if (p) cudaFree(p);
    for (VEC_T *p : lift) if (p) cudaFree(p);
    for (auto &sl : wind) for (auto &t : sl) free_tex(t);
    free_tex(vol);
    free_tex(topo);
    return 0;
}

}  // namespace

extern "C" int ref_run_opt(ref_opt_args *a) {
    a->message[0] = 0;
    if (a->n < 2) {
        snprintf(a->message, sizeof a->message, "the reference's launch shape needs at least 2 particles");
        return 1;
    }
    if (a->n_volumes > 1 || a->n_constants > 4) {
        snprintf(a->message, sizeof a->message, "at most one volume and four constants");
        return 1;
    }
    for (const OptEntry &v : kOpt) {
        if (v.dim == a->dim && v.integrator == a->integrator && v.border == a->border_mode &&
            v.curvature == a->curvature_mode && v.abort_mode == a->abort_mode && v.uplift == a->uplift_mode &&
            v.windfield == a->windfield_mode && v.constants == a->constants_mode && v.volume == a->volume_mode &&
            v.topo == a->use_topography && v.reverse == a->reverse && v.sphere == a->use_sphere &&
            v.comp == a->comp_additional)
            return a->dim == 2 ? run_opt<Vec2>(a, reinterpret_cast<OptLaunch<Vec2>>(v.fn))
                               : run_opt<Vec3>(a, reinterpret_cast<OptLaunch<Vec3>>(v.fn));
    }
    snprintf(a->message, sizeof a->message, "no instantiated reference variant for these settings");
    return 2;
}

extern "C" int ref_run(ref_args *a) {
    a->message[0] = 0;
    if (a->n < 2) {
        snprintf(a->message, sizeof a->message, "the reference's launch shape needs at least 2 particles");
        return 1;
    }
    return a->variant == 0 ? run<Vec2>(a) : run<Vec3>(a);
}
