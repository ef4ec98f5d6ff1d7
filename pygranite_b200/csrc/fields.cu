// fields.cu — native loaders: analytic windfields evaluated on the device (gr_field_*,
// include/granite_b200.h).
//
// The reference feeds every snapshot through a Python DataLoader that returns numpy arrays
// (source/granite/DataLoader.hpp:26-81, TrajectoryIntegrator.cpp:146-360).  For synthetic
// fields this evaluates each snapshot on the GPU instead and hands the planes to the engine's
// device-pointer load, so a run needs no host snapshot memory and no Python in its loop.
// Arithmetic is float64 (no contraction besides the explicit fma of the Fourier sums), rounded
// to float32 at the end.  The double gyre follows the host generator's operation order; the
// Fourier field is, like the host generator, a separable product of per-axis plane-wave factors
// (association order differs, so the two agree to float64 rounding, not bit for bit).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <memory>
#include <string>

#include "../../include/granite_b200.h"
#include "engine_graph.h"
#include "host_util.h"

using namespace granite_b200;

struct gr_field {
    int kind = 0;                      // 0 double gyre, 1 Fourier modes
    int dim = 2;
    int device = 0;
    int64_t nz = 1, ny = 0, nx = 0, nodes = 0;
    double snapshot_dt = 1.0;
    int64_t n_snap = 0;
    // double gyre
    double A = 0, eps = 0, omega = 0, lx = 0, ly = 0;
    // Fourier modes
    int modes = 0;
    double spacing[3]{};               // per axis, grid order (z, y, x) / (y, x)
    DevBuf<double> k, amp, phase, om, scale;
    DevBuf<double2> fac_x, fac_y, fac_z;   // exp(i k_a x_i) per (component, mode) and node index
    DevBuf<double2> coef;              // amp e^{i (phase - omega t)} of the current snapshot
    DevBuf<float> planes;              // dim planes of the current snapshot
    int64_t holds = -1;                // snapshot in `planes`
    cudaStream_t stream = nullptr;
    ~gr_field() {
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

int ffail(int code, const std::string &msg) {
    set_last_error(msg.c_str());
    return code;
}

#define FUSER(msg) ffail(GR_ERR_USER, std::string("ERROR < USER INPUT | ") + (msg) + " >")

#define FK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t err_ = (call);                                                                 \
        if (err_ != cudaSuccess) {                                                                 \
            char buf_[256];                                                                        \
            snprintf(buf_, sizeof buf_, "ERROR < RUNTIME | CUDA error | %s : %s, line %d >",       \
                     cudaGetErrorString(err_), __FILE__, __LINE__);                                \
            return ffail(GR_ERR_RUNTIME, buf_);                                                    \
        }                                                                                          \
    } while (0)

// u = -pi A sin(pi f) cos(pi y), v = pi A cos(pi f) sin(pi y) df/dx,
// f = a x^2 + b x, a = eps sin(w t), b = 1 - 2 eps sin(w t)
__global__ void double_gyre_kernel(double A, double eps, double omega, double t, int64_t ny, int64_t nx,
                                   double dx, double dy, float *__restrict__ u, float *__restrict__ v) {
    const int64_t nodes = nx * ny;
    const double pi = 3.141592653589793;
    const double s = sin(omega * t);
    const double a = eps * s, b = 1.0 - 2.0 * eps * s;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = (double)(i % nx) * dx, y = (double)(i / nx) * dy;
        const double f = a * x * x + b * x;
        const double dfdx = 2.0 * a * x + b;
        u[i] = (float)(-pi * A * sin(pi * f) * cos(pi * y));
        v[i] = (float)(pi * A * cos(pi * f) * sin(pi * y) * dfdx);
    }
}

// Per-axis plane-wave factors, time-independent: fac[cm][i] = exp(i k_cm,a x_i), x_i = i * spacing
// along grid axis a (k holds each mode's wave vector in grid order, z y x / y x).
__global__ void fourier_factors_kernel(const double *__restrict__ k, int dim, int axis, int64_t cms, int64_t n,
                                       double spacing, double2 *__restrict__ fac) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < cms * n; j += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cm = j / n, i = j % n;
        double sn, cs;
        sincos(k[cm * dim + axis] * ((double)i * spacing), &sn, &cs);
        fac[j] = make_double2(cs, sn);
    }
}

// The snapshot's mode coefficients: coef[cm] = amp_cm exp(i (phase_cm - omega_cm t)).
__global__ void fourier_coef_kernel(const double *__restrict__ amp, const double *__restrict__ phase,
                                    const double *__restrict__ om, int64_t cms, double t, double2 *__restrict__ coef) {
    for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < cms; j += (int64_t)gridDim.x * blockDim.x) {
        double sn, cs;
        sincos(phase[j] - om[j] * t, &sn, &cs);
        coef[j] = make_double2(amp[j] * cs, amp[j] * sn);
    }
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

constexpr int kFieldThreads = 128;   // x positions per block
constexpr int kFieldRows = 8;        // grid rows (consecutive (z, y) pairs) per block
constexpr int kModeChunk = 64;       // modes whose row coefficients are staged at once

// component c = scale_c Re sum_m (coef_cm fz_cm[iz] fy_cm[iy]) fx_cm[ix]: the plane waves as a
// rank-`modes` separable product, so a node costs two multiply-adds per mode instead of a
// cosine.  The row coefficients (everything but fx) of a chunk of modes are staged in shared
// memory for the block's kFieldRows rows; each thread keeps one x position's sums for all of them.
__global__ void __launch_bounds__(kFieldThreads) fourier_rows_kernel(
        const double2 *__restrict__ fx, const double2 *__restrict__ fy, const double2 *__restrict__ fz,
        const double2 *__restrict__ coef, const double *__restrict__ scale, int dim, int modes, int64_t nz,
        int64_t ny, int64_t nx, float *__restrict__ out) {
    __shared__ double2 w[kModeChunk][kFieldRows];
    const int64_t rows = nz * ny, nodes = rows * nx;
    const int64_t ix = (int64_t)blockIdx.x * kFieldThreads + threadIdx.x;
    const bool in_x = ix < nx;
    for (int64_t row0 = (int64_t)blockIdx.y * kFieldRows; row0 < rows; row0 += (int64_t)gridDim.y * kFieldRows) {
        for (int c = 0; c < dim; ++c) {
            double acc[kFieldRows];
#pragma unroll
            for (int r = 0; r < kFieldRows; ++r) acc[r] = 0.0;
            for (int m0 = 0; m0 < modes; m0 += kModeChunk) {
                const int mc = min(kModeChunk, modes - m0);
                __syncthreads();   // the previous chunk's coefficients are no longer read
                for (int j = threadIdx.x; j < mc * kFieldRows; j += kFieldThreads) {
                    const int mm = j / kFieldRows, r = j % kFieldRows;
                    const int64_t row = row0 + r, cm = (int64_t)c * modes + m0 + mm;
                    double2 v = make_double2(0.0, 0.0);
                    if (row < rows) {
                        v = coef[cm];
                        if (dim == 3) v = cmul(v, fz[cm * nz + row / ny]);
                        v = cmul(v, fy[cm * ny + row % ny]);
                    }
                    w[mm][r] = v;
                }
                __syncthreads();
                if (in_x) {
                    for (int mm = 0; mm < mc; ++mm) {
                        const double2 e = fx[((int64_t)c * modes + m0 + mm) * nx + ix];
#pragma unroll
                        for (int r = 0; r < kFieldRows; ++r) acc[r] = fma(-w[mm][r].y, e.y, fma(w[mm][r].x, e.x, acc[r]));
                    }
                }
            }
            if (in_x) {
#pragma unroll
                for (int r = 0; r < kFieldRows; ++r)
                    if (row0 + r < rows) out[(int64_t)c * nodes + (row0 + r) * nx + ix] = (float)(acc[r] * scale[c]);
            }
        }
    }
}

int generate(gr_field *f, int64_t snapshot) {
    if (snapshot < 0 || snapshot >= f->n_snap) return FUSER("snapshot index out of range");
    if (f->holds == snapshot) return GR_OK;
    FK(cudaSetDevice(f->device));
    const double t = (double)snapshot * f->snapshot_dt;
    const int threads = 256, blocks = grid_for(f->nodes, threads);
    if (f->kind == 0) {
        double_gyre_kernel<<<blocks, threads, 0, f->stream>>>(f->A, f->eps, f->omega, t, f->ny, f->nx,
                                                              f->lx / (double)f->nx, f->ly / (double)f->ny,
                                                              f->planes.p, f->planes.p + f->nodes);
    } else {
        const int64_t cms = (int64_t)f->dim * f->modes;
        fourier_coef_kernel<<<grid_for(cms, 256), 256, 0, f->stream>>>(f->amp.p, f->phase.p, f->om.p, cms, t, f->coef.p);
        FK(cudaGetLastError());
        const int64_t groups = (f->nz * f->ny + kFieldRows - 1) / kFieldRows;
        const dim3 grid((unsigned)((f->nx + kFieldThreads - 1) / kFieldThreads), (unsigned)std::min<int64_t>(groups, 65535));
        fourier_rows_kernel<<<grid, kFieldThreads, 0, f->stream>>>(f->fac_x.p, f->fac_y.p, f->fac_z.p, f->coef.p,
                                                                   f->scale.p, f->dim, f->modes, f->nz, f->ny, f->nx,
                                                                   f->planes.p);
    }
    FK(cudaGetLastError());
    FK(cudaStreamSynchronize(f->stream));
    f->holds = snapshot;
    return GR_OK;
}

int finish_create(gr_field *f) {
    FK(cudaSetDevice(f->device));
    FK(cudaStreamCreateWithFlags(&f->stream, cudaStreamNonBlocking));
    FK(f->planes.alloc((size_t)f->nodes * f->dim));
    return GR_OK;
}

}  // namespace

extern "C" {

int gr_field_double_gyre(double A, double eps, double omega, int64_t ny, int64_t nx, double lx, double ly,
                         double snapshot_dt, int64_t n_snapshots, int32_t device, gr_field **out) {
    if (!out) return FUSER("null argument");
    *out = nullptr;
    if (nx < 1 || ny < 1 || nx * ny > (int64_t(1) << 34)) return FUSER("Invalid dataset was provided. Empty grid.");
    if (n_snapshots < 1 || !(snapshot_dt > 0.0) || !(lx > 0.0) || !(ly > 0.0)) return FUSER("invalid field parameters");
    auto f = std::make_unique<gr_field>();
    f->kind = 0;
    f->dim = 2;
    f->device = device;
    f->ny = ny; f->nx = nx; f->nz = 1; f->nodes = nx * ny;
    f->A = A; f->eps = eps; f->omega = omega; f->lx = lx; f->ly = ly;
    f->snapshot_dt = snapshot_dt;
    f->n_snap = n_snapshots;
    const int rc = finish_create(f.get());
    if (rc) return rc;
    *out = f.release();
    return GR_OK;
}

int gr_field_fourier(int32_t dim, const int64_t *shape, const double *spacing, int32_t n_modes, const double *k,
                     const double *amp, const double *phase, const double *omega, const double *scale,
                     double snapshot_dt, int64_t n_snapshots, int32_t device, gr_field **out) {
    if (!out || !shape || !spacing || !k || !amp || !phase || !omega || !scale) return FUSER("null argument");
    *out = nullptr;
    if (dim != 2 && dim != 3) return FUSER("Invalid Space.");
    if (n_modes < 1 || n_modes > 4096) return FUSER("invalid mode count");
    if (n_snapshots < 1 || !(snapshot_dt > 0.0)) return FUSER("invalid field parameters");
    int64_t nodes = 1;
    for (int d = 0; d < dim; ++d) {
        if (shape[d] < 1 || shape[d] > (int64_t(1) << 30)) return FUSER("Invalid dataset was provided. Empty grid.");
        nodes *= shape[d];
    }
    if (nodes > (int64_t(1) << 34)) return FUSER("Invalid dataset was provided. Grid too large.");
    auto f = std::make_unique<gr_field>();
    f->kind = 1;
    f->dim = dim;
    f->device = device;
    f->nz = dim == 3 ? shape[0] : 1;
    f->ny = shape[dim - 2];
    f->nx = shape[dim - 1];
    f->nodes = nodes;
    for (int d = 0; d < dim; ++d) f->spacing[d] = spacing[d];
    f->modes = n_modes;
    f->snapshot_dt = snapshot_dt;
    f->n_snap = n_snapshots;
    int rc = finish_create(f.get());
    if (rc) return rc;
    const size_t cm = (size_t)dim * n_modes;
    FK(f->k.alloc(cm * dim)); FK(f->amp.alloc(cm)); FK(f->phase.alloc(cm)); FK(f->om.alloc(cm));
    FK(f->scale.alloc((size_t)dim));
    FK(cudaMemcpy(f->k.p, k, cm * dim * sizeof(double), cudaMemcpyHostToDevice));
    FK(cudaMemcpy(f->amp.p, amp, cm * sizeof(double), cudaMemcpyHostToDevice));
    FK(cudaMemcpy(f->phase.p, phase, cm * sizeof(double), cudaMemcpyHostToDevice));
    FK(cudaMemcpy(f->om.p, omega, cm * sizeof(double), cudaMemcpyHostToDevice));
    FK(cudaMemcpy(f->scale.p, scale, (size_t)dim * sizeof(double), cudaMemcpyHostToDevice));
    // the per-axis factors of every mode (time-independent)
    FK(f->coef.alloc(cm));
    FK(f->fac_x.alloc(cm * (size_t)f->nx));
    FK(f->fac_y.alloc(cm * (size_t)f->ny));
    if (dim == 3) FK(f->fac_z.alloc(cm * (size_t)f->nz));
    struct Axis { DevBuf<double2> *fac; int axis; int64_t n; };
    const Axis axes[3] = {{&f->fac_x, dim - 1, f->nx}, {&f->fac_y, dim - 2, f->ny}, {&f->fac_z, 0, f->nz}};
    for (int a = 0; a < dim; ++a) {
        const int64_t total = (int64_t)cm * axes[a].n;
        fourier_factors_kernel<<<grid_for(total, 256), 256, 0, f->stream>>>(f->k.p, dim, axes[a].axis, (int64_t)cm,
                                                                             axes[a].n, f->spacing[axes[a].axis],
                                                                             axes[a].fac->p);
        FK(cudaGetLastError());
    }
    FK(cudaStreamSynchronize(f->stream));
    *out = f.release();
    return GR_OK;
}

int gr_field_load(gr_field *f, gr_engine *e, int64_t snapshot) {
    if (!f || !e) return FUSER("null argument");
    if (engine_device(e) != f->device) return FUSER("the field and the engine use different devices");
    int rc = generate(f, snapshot);
    if (rc) return rc;
    const float *planes[3] = {f->planes.p, f->planes.p + f->nodes, f->planes.p + 2 * f->nodes};
    return gr_load_windfield_device(e, snapshot, planes, f->dim, f->nz, f->ny, f->nx);
}

int gr_field_loader(void *user, gr_engine *e, int64_t snapshot) {
    gr_field *f = static_cast<gr_field *>(user);
    if (!f) return -1;
    if (snapshot >= f->n_snap) return 0;
    return gr_field_load(f, e, snapshot) == GR_OK ? 1 : -1;
}

int gr_field_snapshot(gr_field *f, int64_t snapshot, float *out, int64_t cap) {
    if (!f || !out) return FUSER("null argument");
    if (cap < f->nodes * f->dim) return FUSER("Output buffer too small.");
    int rc = generate(f, snapshot);
    if (rc) return rc;
    FK(cudaMemcpy(out, f->planes.p, (size_t)f->nodes * f->dim * sizeof(float), cudaMemcpyDeviceToHost));
    return GR_OK;
}

void gr_field_destroy(gr_field *f) { delete f; }

}  // extern "C"
