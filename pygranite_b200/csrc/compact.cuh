// compact.cuh — retirement of aborted particles and spatial re-sorting of the live ones.
//
// Between launches the live particles are counting-sorted by the Morton rank of the grid
// brick they sit in (4x4x2 nodes in 3D, 4x4 in 2D), so a warp samples neighbouring cells
// and the gathers of one warp share cache lines.  Aborted particles go to a separate
// retired store and are never launched again; the records they would have written later
// repeat their frozen state, substituted when the history is read (RowFill, engine.cu).  Per-particle arithmetic does
// not depend on the order, so results stay bit-identical.
//
// Kernels are static: every translation unit that includes this header owns its instances.
//
// One pass: bin (key + warp-aggregated histogram) -> two-level exclusive scan -> rank
// (destination of every source slot, written as a permutation) -> gather (coalesced writes
// of every state array) -> commit (counts).
#pragma once

#include <cstdint>

#include "granite_kernels.cuh"

namespace granite_b200 {

constexpr int SCAN_CHUNK = 1024;   // bins per block of the first scan level

struct StateView {
    float *px, *py, *pz, *qx, *qy, *qz, *kx, *ky, *kz, *lx, *ly, *lz;
    float *length, *tc, *curv, *volc, *cmpc;
    float4 *vlast;    // deferred volume / expression inputs (KParams::vlast), or null
    int32_t *status, *id, *retire, *life, *birth;
    int64_t stride;   // per-array stride of volc / cmpc
};

struct CompactParams {
    StateView src, dst, ret;
    int32_t *key;              // bin of each active slot
    int32_t *hist;             // nbins + 1 counters -> offsets within the chunk -> cursors
    int32_t *chunk;            // per-chunk sums -> chunk base offsets
    int32_t *perm;             // destination slot -> source slot
    const int32_t *bintab;     // brick linear index -> Morton rank
    int32_t *n_act;            // active count (device)
    int32_t *n_new;            // live count after the pass (device)
    int32_t *n_ret;            // retired count (device)
    float off[3], inv_scale[3];
    int32_t nx, ny, nz, dim;
    int32_t bx, by, bz, nbx, nby, nbz, nbins;
    int32_t nvol, nexpr, curv_prev, compensated, fast_curv, abort_on, curv_on, curv_ind;
    int32_t rec_now;           // first record index not yet written
    int32_t k_end;             // steps run so far: a particle whose lifetime is over retires
    int32_t ret_by_id;         // 1: retired particles go to slot id of `ret` (final state only)
};

__device__ __forceinline__ int32_t bin_of(const CompactParams &C, int64_t i) {
    // retired bin (last): aborted, or its lifetime is over (status stays Time)
    if (C.src.status[i] != 0 || (C.src.life && C.src.life[i] <= C.k_end)) return C.nbins;
    const float ax = (C.src.px[i] - C.off[0]) * C.inv_scale[0];
    const float ay = (C.src.py[i] - C.off[1]) * C.inv_scale[1];
    const int ix = (int)fminf(fmaxf(floorf(ax), 0.f), (float)(C.nx - 1));
    const int iy = (int)fminf(fmaxf(floorf(ay), 0.f), (float)(C.ny - 1));
    int iz = 0;
    if (C.dim == 3) {
        const float az = (C.src.pz[i] - C.off[2]) * C.inv_scale[2];
        iz = (int)fminf(fmaxf(floorf(az), 0.f), (float)(C.nz - 1));
    }
    return C.bintab[((iz / C.bz) * C.nby + iy / C.by) * C.nbx + ix / C.bx];
}

// key + histogram; lanes of a warp with the same key add once (sorted input: mostly one key per warp)
static __global__ void bin_kernel(const __grid_constant__ CompactParams C) {
    const int64_t n = *C.n_act;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        const bool ok = i < n;
        const int32_t k = ok ? bin_of(C, i) : -1;
        if (ok) C.key[i] = k;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        const int leader = __ffs(peers) - 1;
        if (ok && (int)(threadIdx.x & 31) == leader) atomicAdd(C.hist + k, __popc(peers));
    }
}

// level 1: exclusive scan inside chunks of SCAN_CHUNK bins; chunk totals to C.chunk
static __global__ void __launch_bounds__(SCAN_CHUNK) scan_chunks_kernel(const __grid_constant__ CompactParams C) {
    __shared__ int32_t warp_sum[SCAN_CHUNK / 32];
    const int nb = C.nbins + 1;
    const int b = blockIdx.x * SCAN_CHUNK + threadIdx.x;
    const int32_t v = b < nb ? C.hist[b] : 0;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[wid] = x;
    __syncthreads();
    if (wid == 0) {
        int32_t s = warp_sum[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sum[lane] = s;   // inclusive over warps
    }
    __syncthreads();
    const int32_t incl = x + (wid > 0 ? warp_sum[wid - 1] : 0);
    if (b < nb) C.hist[b] = incl - v;
    if (threadIdx.x == SCAN_CHUNK - 1) C.chunk[blockIdx.x] = incl;
}

// level 2: exclusive scan of the chunk totals (one block); n_new = start of the retired bin
static __global__ void __launch_bounds__(1024) scan_top_kernel(const __grid_constant__ CompactParams C, int nchunks) {
    __shared__ int32_t part[1024];
    const int per = (nchunks + 1023) / 1024;
    const int c0 = threadIdx.x * per, c1 = min(nchunks, c0 + per);
    int32_t s = 0;
    for (int c = c0; c < c1; ++c) s += C.chunk[c];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        const int32_t y = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0;
        __syncthreads();
        part[threadIdx.x] += y;
        __syncthreads();
    }
    int32_t run = part[threadIdx.x] - s;
    for (int c = c0; c < c1; ++c) {
        const int32_t t = C.chunk[c];
        C.chunk[c] = run;
        run += t;
    }
    __syncthreads();
    if (threadIdx.x == 0) *C.n_new = C.hist[C.nbins] + C.chunk[C.nbins / SCAN_CHUNK];
}

// destination of every source slot, as a permutation dest -> source
static __global__ void rank_kernel(const __grid_constant__ CompactParams C) {
    const int64_t n = *C.n_act;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n; base += stride) {
        const int64_t i = base + threadIdx.x;
        const bool ok = i < n;
        const int32_t k = ok ? C.key[i] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, k);
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(peers) - 1;
        int32_t first = 0;
        if (ok && lane == leader) first = atomicAdd(C.hist + k, __popc(peers));
        first = __shfl_sync(0xffffffffu, first, leader);
        if (ok) {
            const int32_t d = C.chunk[k / SCAN_CHUNK] + first + __popc(peers & ((1u << lane) - 1));
            C.perm[d] = (int32_t)i;
        }
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
    if (S.vlast) D.vlast[d] = S.vlast[i];
    D.status[d] = S.status[i];
    D.id[d] = S.id[i];
    if (S.life) D.life[d] = S.life[i];
    if (S.birth) D.birth[d] = S.birth[i];
}

__device__ __forceinline__ void move_retired(const CompactParams &C, int64_t i, int64_t r) {
    const StateView &S = C.src, &R = C.ret;
    if (C.ret_by_id) {   // final state straight into the result slot of the particle
        const int64_t id = S.id[i];
        R.px[id] = S.px[i]; R.py[id] = S.py[i];
        if (C.dim == 3) R.pz[id] = S.pz[i];
        R.status[id] = S.status[i];
        return;
    }
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

// coalesced writes in destination order; the scattered reads hit L2
static __global__ void gather_kernel(const __grid_constant__ CompactParams C) {
    const int64_t n = *C.n_act, live = *C.n_new, base = *C.n_ret;
    for (int64_t d = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; d < n; d += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = C.perm[d];
        if (d < live) move_live(C, i, d);
        else move_retired(C, i, base + (d - live));
    }
}

static __global__ void commit_kernel(const __grid_constant__ CompactParams C) {
    *C.n_ret += *C.n_act - *C.n_new;
    *C.n_act = *C.n_new;
}

}  // namespace granite_b200
