// compact.cuh — retirement of aborted particles and spatial re-sorting of the live ones.
//
// Between launches the live particles are counting-sorted by the Morton rank of the grid
// brick they sit in (4x4x2 nodes in 3D, 4x4 in 2D), so a warp samples neighbouring cells
// and the gathers of one warp share cache lines.  Aborted particles go to a separate
// retired store and are never launched again; the records they would have written later
// are filled from their frozen state at the end of the run.  Per-particle arithmetic does
// not depend on the order, so results stay bit-identical.
#pragma once

#include <cstdint>

#include "granite_kernels.cuh"

namespace granite_b200 {

struct StateView {
    float *px, *py, *pz, *qx, *qy, *qz, *kx, *ky, *kz, *lx, *ly, *lz;
    float *length, *tc, *curv, *volc, *cmpc;
    int32_t *status, *id, *retire;
    int64_t stride;   // per-array stride of volc / cmpc
};

struct CompactParams {
    StateView src, dst, ret;
    int32_t *key;              // bin of each active slot
    int32_t *hist;             // nbins + 1 counters -> cursors
    const int32_t *bintab;     // brick linear index -> Morton rank
    int32_t *n_act;            // active count (device)
    int32_t *n_new;            // live count after the pass (device)
    int32_t *n_ret;            // retired count (device)
    float off[3], inv_scale[3];
    int32_t nx, ny, nz, dim;
    int32_t bx, by, bz, nbx, nby, nbz, nbins;
    int32_t nvol, nexpr, curv_prev, compensated, fast_curv, abort_on, curv_on, curv_ind;
    int32_t rec_now;           // first record index not yet written
};

__global__ void bin_kernel(const __grid_constant__ CompactParams C) {
    const int64_t n = *C.n_act;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t k = C.nbins;   // retired bin, last
        if (C.src.status[i] == 0) {
            const float ax = (C.src.px[i] - C.off[0]) * C.inv_scale[0];
            const float ay = (C.src.py[i] - C.off[1]) * C.inv_scale[1];
            int ix = (int)fminf(fmaxf(floorf(ax), 0.f), (float)(C.nx - 1));
            int iy = (int)fminf(fmaxf(floorf(ay), 0.f), (float)(C.ny - 1));
            int iz = 0;
            if (C.dim == 3) {
                const float az = (C.src.pz[i] - C.off[2]) * C.inv_scale[2];
                iz = (int)fminf(fmaxf(floorf(az), 0.f), (float)(C.nz - 1));
            }
            const int b = ((iz / C.bz) * C.nby + iy / C.by) * C.nbx + ix / C.bx;
            k = C.bintab[b];
        }
        C.key[i] = k;
        atomicAdd(C.hist + k, 1);
    }
}

// Exclusive scan of the nbins + 1 counters in one block; n_new = start of the retired bin.
__global__ void __launch_bounds__(1024) scan_kernel(const __grid_constant__ CompactParams C) {
    __shared__ int32_t part[1024];
    const int nb = C.nbins + 1;
    const int per = (nb + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per, b1 = min(nb, b0 + per);
    int32_t s = 0;
    for (int b = b0; b < b1; ++b) s += C.hist[b];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
        const int32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    int32_t run = part[threadIdx.x] - s;   // exclusive prefix of this chunk
    for (int b = b0; b < b1; ++b) {
        const int32_t c = C.hist[b];
        C.hist[b] = run;
        if (b == C.nbins) *C.n_new = run;
        run += c;
    }
}

__device__ __forceinline__ void move_live(const CompactParams &C, int64_t i, int64_t d) {
    const StateView &S = C.src, &D = C.dst;
    D.px[d] = S.px[i]; D.py[d] = S.py[i];
    if (C.dim == 3) D.pz[d] = S.pz[i];
    if (C.curv_prev) { D.qx[d] = S.qx[i]; D.qy[d] = S.qy[i]; if (C.dim == 3) D.qz[d] = S.qz[i]; }
    if (C.compensated) { D.kx[d] = S.kx[i]; D.ky[d] = S.ky[i]; if (C.dim == 3) D.kz[d] = S.kz[i]; }
    if (C.fast_curv) { D.lx[d] = S.lx[i]; D.ly[d] = S.ly[i]; if (C.dim == 3) D.lz[d] = S.lz[i]; }
    if (C.abort_on) D.length[d] = S.length[i];
    if (C.curv_on) D.tc[d] = S.tc[i];
    if (C.curv_ind) D.curv[d] = S.curv[i];
    for (int k = 0; k < C.nvol; ++k) D.volc[k * D.stride + d] = S.volc[k * S.stride + i];
    for (int k = 0; k < C.nexpr; ++k) D.cmpc[k * D.stride + d] = S.cmpc[k * S.stride + i];
    D.status[d] = S.status[i];
    D.id[d] = S.id[i];
}

__device__ __forceinline__ void move_retired(const CompactParams &C, int64_t i, int64_t r) {
    const StateView &S = C.src, &R = C.ret;
    R.px[r] = S.px[i]; R.py[r] = S.py[i];
    if (C.dim == 3) R.pz[r] = S.pz[i];
    if (C.abort_on) R.length[r] = S.length[i];
    if (C.curv_on) R.tc[r] = S.tc[i];
    if (C.curv_ind) R.curv[r] = S.curv[i];
    for (int k = 0; k < C.nvol; ++k) R.volc[k * R.stride + r] = S.volc[k * S.stride + i];
    for (int k = 0; k < C.nexpr; ++k) R.cmpc[k * R.stride + r] = S.cmpc[k * S.stride + i];
    R.status[r] = S.status[i];
    R.id[r] = S.id[i];
    R.retire[r] = C.rec_now;
}

__global__ void scatter_kernel(const __grid_constant__ CompactParams C) {
    const int64_t n = *C.n_act, live = *C.n_new, base = *C.n_ret;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t d = atomicAdd(C.hist + C.key[i], 1);
        if (d < live) move_live(C, i, d);
        else move_retired(C, i, base + (d - live));
    }
}

__global__ void commit_kernel(const __grid_constant__ CompactParams C) {
    *C.n_ret += *C.n_act - *C.n_new;
    *C.n_act = *C.n_new;
}

}  // namespace granite_b200
