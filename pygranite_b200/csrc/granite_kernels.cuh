// granite_kernels.cuh — sm_100a device code of the trajectory step path.
//
// One thread owns one particle.  A launch advances its particle through a range of steps
// (one or more snapshot windows) with the particle state in registers; the reference
// instead launches `integrate` once per step on a single 512-thread block and
// double-buffers AoS positions through global memory (TrajectoryIntegrator.tpp:108-457,
// 790-796, 978-984).  Per step the uniform data (time weights, save slots, ring slots)
// comes from a small device schedule.
//
// Arithmetic follows one fixed operation order, spelled out with __fmaf_rn and compiled
// with --fmad=false, so the float32 oracle build reproduces it bit for bit.  Wind is
// stored node-major: float4 {u,v,w,0} (3D) or float2 {u,v} (2D) per node for float32,
// four / two 16-bit values per node for bf16 / fp16.  Hardware texture filtering (8-bit
// weights, TrajectoryIntegrator.cpp:503-505) is replaced by float32 interpolation.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#ifdef __CUDACC_RTC__
// run-time compilation of the deferred volume / expression kernel (jit.cu): no host headers
typedef signed char int8_t;
typedef short int16_t;
typedef int int32_t;
typedef long long int64_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
namespace std {
template <class A, class B> struct is_same { static constexpr bool value = false; };
template <class A> struct is_same<A, A> { static constexpr bool value = true; };
}  // namespace std
#else
#include <cstdint>
#include <type_traits>
#endif

#include "expr.h"

namespace granite_b200 {

constexpr int GR_MAX_VOL = 8;
constexpr int GR_MAX_EXPR = 4;
constexpr int GR_MAX_CON = 4;

// Compile-time feature sets of the step kernel.  FT_GENERIC honours every runtime option.  A
// lean variant (FT_LEAN) is picked by the host (kernel_features in advance.h) when the launch has
// no uplift, length abort, topography, sphere coordinates, loop borders, per-step alive counts
// or 1/256 filter weights, and curvature Off or Total; FT_CURV / FT_EXTRAS say whether it keeps total curvature and volume
// / expression values, FT_COMP Kahan-compensated positions (instantiated without extras: the
// precision form).  FT_DEFER (with FT_LEAN, instead of FT_EXTRAS) leaves the volume / expression
// values to deferred_extras_kernel after the launch: the step kernel only stores each moved step's
// stage-averaged velocity and step index, and hands them to the record at a save step.  The lean
// variants drop the dead state from registers; their arithmetic is the generic variant's.
constexpr int FT_GENERIC = 0, FT_LEAN = 1, FT_CURV = 2, FT_EXTRAS = 4, FT_COMP = 8, FT_DEFER = 16;

// Step-schedule flags.
constexpr int SF_SAVE = 1;       // position / info record after this step
constexpr int SF_TIME_POS = 2;   // data.Time > 0 at the start of the step
constexpr int SF_CURV_REC = 4;   // curvature record after this step (IndividualAndTotal)

struct StepEntry {
    float t0, t1, t2;      // time weights of the RK4 stages (t1 also for k3)
    int32_t flags;
    int32_t rec, crec, irec;
    int32_t slot_back, slot_front;   // ring slots of the window's snapshots
    int32_t pad[3];
};

struct KParams {
    // geometry (TrajectoryIntegrator.tpp:521-574)
    float inv_scale[3], off[3], dom[3], scale[3];
    int32_t nx, ny, nz, dim;
    float fn[3];                  // nx, ny, nz as floats (the upper clamp of the window pair's cells)
    // ring buffers: slot s of quantity q starts at base + s * stride
    const void *wind;
    int64_t wind_stride;          // bytes per slot
    const void *pair;             // window-pair buffer of the launch's window (pair layouts)
    int32_t pnx, pnxy;            // window pair: padded row length (nx + 3) and plane size
                                  // ((nx + 3) * (ny + 3)); node (x, y, z) at
                                  // (z + 1) * pnxy + (y + 1) * pnx + (x + 1): zeros outside the
                                  // grid in 3D, the clamped edge node in 2D
    const float *vol;             // [slot][8][plane]
    int64_t vol_plane;            // floats per plane
    const float *cons;            // [slot][4][n_total]
    const float *lift;            // [slot][n_total * dim]
    const float *topo;            // (ny, nx)
    // particle state, slot order
    float *px, *py, *pz;          // position
    float *qx, *qy, *qz;          // previous position (curvature pm1)
    float *kx, *ky, *kz;          // Kahan compensation
    float *lx, *ly, *lz;          // last direction (FastTotal curvature)
    int32_t *status;
    float *length, *tc, *curv;
    float *volc;                  // [8][n_state]
    float *cmpc;                  // [4][n_state]
    float4 *vlast;                // FT_DEFER: (stage-averaged velocity, step index as int bits) of
                                  // each slot's last moved step; index -1: no step since the values
                                  // were last evaluated (or handed to a record)
    float4 *vrec;                 // FT_DEFER: [2 i] position, [2 i + 1] vlast as of the launch's
                                  // save step, for its record
    const int32_t *id;            // original particle index
    int64_t n;                    // particles in this launch (prefix of the state arrays)
    const int32_t *n_dev;         // if set: live prefix length on the device (<= n)
    const int32_t *life;          // if set: steps each slot may run (batched sets of uneven lifetime)
    const int32_t *birth;         // if set: first step each slot runs (served requests joining mid-window)
    int32_t grid_stride;          // 1: persistent grid striding over the live prefix
    int64_t n_state;              // stride of volc / cmpc
    int64_t n_total;              // original particle count (history / constants stride)
    // history, record-major: one row of n_total particles per record, so the rows a launch
    // writes are whole in L2 before they reach DRAM (the fetch transposes them)
    float *hpos;                  // [(rec * n_total + id) * dim + d]
    float *hcurv;                 // [crec * n_total + id]
    float *hvol;                  // [(k * Li + irec) * n_total + id]
    float *hcmp;                  // [(e * Li + irec) * n_total + id]
    int64_t L, Lc, Li;
    // schedule
    const StepEntry *sched;
    int32_t s0, s1;
    // options (runtime-uniform)
    float h, hh, sixth, max_length, sphere_radius;
    float inv_2h, inv_hh;         // 1 / (2 h) and 1 / (h h), rounded to float (curvature differences)
    int32_t wind_dynamic, dyn_any, border_mode, curvature_mode, abort_mode, uplift_mode;
    int32_t constants_mode, volume_mode, reverse, sphere, topography, compensated;
    int32_t nvol, ncon, nexpr;
    int32_t filter_weights;       // 1: interpolation fractions rounded to the nearest 1/256
    const Program *prog;          // [4]
    unsigned long long *counters; // [0] particle-steps, [1] alive at the end of the launch
    unsigned *alive_at;           // if set: [step - s0][32 shards] particles alive after each step
};

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ float lerp_(float a, float b, float t) { return __fmaf_rn(t, b - a, a); }

// Texture coordinate -> cell index and fraction.  Coordinates are clamped to [-2, n+1]
// first; every corner outside the grid is border (3D) or clamped (2D), so the clamp never
// changes a value and keeps the integer conversion in range.
// fw = 1 rounds the fraction to the nearest 1/256, the 8-bit weights of the texture unit the
// reference filters with (CUDA Programming Guide, linear filtering); 0 keeps it exact.
__device__ __forceinline__ void cell(float a, int n, int fw, int &i, float &f) {
    a = fminf(fmaxf(a, -2.0f), (float)(n + 1));
    const float fl = floorf(a);
    i = (int)fl;
    f = a - fl;
    if (fw) f = floorf(f * 256.0f + 0.5f) * (1.0f / 256.0f);
}

template <typename W> struct Store;

template <> struct Store<float> {
    // 3D node {u, v, w, 0}
    static __device__ __forceinline__ void load3(const void *base, int32_t idx, float &u, float &v, float &w) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(base) + idx);
        u = q.x; v = q.y; w = q.z;
    }
    static __device__ __forceinline__ void load2(const void *base, int32_t idx, float &u, float &v) {
        const float2 q = __ldg(reinterpret_cast<const float2 *>(base) + idx);
        u = q.x; v = q.y;
    }
    static constexpr int bytes3 = 16, bytes2 = 8;
};

template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ void load3(const void *base, int32_t idx, float &u, float &v, float &w) {
        const uint2 q = __ldg(reinterpret_cast<const uint2 *>(base) + idx);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&q.x));
        const float2 b = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&q.y));
        u = a.x; v = a.y; w = b.x;
    }
    static __device__ __forceinline__ void load2(const void *base, int32_t idx, float &u, float &v) {
        const unsigned q = __ldg(reinterpret_cast<const unsigned *>(base) + idx);
        const float2 a = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&q));
        u = a.x; v = a.y;
    }
    static constexpr int bytes3 = 8, bytes2 = 4;
};

template <> struct Store<__half> {
    static __device__ __forceinline__ void load3(const void *base, int32_t idx, float &u, float &v, float &w) {
        const uint2 q = __ldg(reinterpret_cast<const uint2 *>(base) + idx);
        const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&q.x));
        const float2 b = __half22float2(*reinterpret_cast<const __half2 *>(&q.y));
        u = a.x; v = a.y; w = b.x;
    }
    static __device__ __forceinline__ void load2(const void *base, int32_t idx, float &u, float &v) {
        const unsigned q = __ldg(reinterpret_cast<const unsigned *>(base) + idx);
        const float2 a = __half22float2(*reinterpret_cast<const __half2 *>(&q));
        u = a.x; v = a.y;
    }
    static constexpr int bytes3 = 8, bytes2 = 4;
};

// Window-pair layouts: node n holds, component by component, the back snapshot's value followed
// by the front snapshot's: {u_b, u_f, v_b, v_f, w_b, w_f, 0, 0} in 3D (32 bytes float32, 16 bytes
// 16-bit), {u_b, u_f, v_b, v_f} in 2D (16 / 8 bytes).  One load returns both snapshots, and each
// component arrives as a (back, front) pair that the paired float32 instructions of sm_100
// (__ffma2_rn) interpolate in space at once.  Built per window from the ring (pack_kernels.cuh),
// with a border (make_pcell, bil2p_padded).
template <typename W> struct Pair {};

template <typename W> struct IsPair { static constexpr bool value = false; };
template <typename W> struct IsPair<Pair<W>> { static constexpr bool value = true; };

template <> struct Store<Pair<float>> {
    // 3D node: (u_b, u_f), (v_b, v_f), (w_b, w_f), one 256-bit load
    static __device__ __forceinline__ void load3p(const void *base, int32_t idx, float2 (&c)[3]) {
        float r[8];
        const float *p = reinterpret_cast<const float *>(base) + (int64_t)idx * 8;
        asm volatile("ld.global.nc.v8.f32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                     : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
                     : "l"(p));
        c[0] = make_float2(r[0], r[1]); c[1] = make_float2(r[2], r[3]); c[2] = make_float2(r[4], r[5]);
    }
    // 2D node: (u_b, u_f), (v_b, v_f)
    static __device__ __forceinline__ void load2p(const void *base, int32_t idx, float2 (&c)[2]) {
        const float4 q = __ldg(reinterpret_cast<const float4 *>(base) + idx);
        c[0] = make_float2(q.x, q.y); c[1] = make_float2(q.z, q.w);
    }
    static constexpr int bytes3 = 32, bytes2 = 16;
};

template <typename H> struct Store<Pair<H>> {
    // one 32-bit word = (back, front) of one component, converted to a float pair
    static __device__ __forceinline__ float2 cvt(unsigned q) {
        if constexpr (sizeof(H) == 2 && std::is_same<H, __half>::value)
            return __half22float2(*reinterpret_cast<const __half2 *>(&q));
        else
            return __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&q));
    }
    static __device__ __forceinline__ void load2p(const void *base, int32_t idx, float2 (&c)[2]) {
        const uint2 q = __ldg(reinterpret_cast<const uint2 *>(base) + idx);
        c[0] = cvt(q.x); c[1] = cvt(q.y);
    }
    static constexpr int bytes3 = 16, bytes2 = 8;
};

// Trilinear corner weights of one sample: indices and border validity.
struct Cell3 {
    int32_t base;        // node index of corner (ix, iy, iz), clamped into the grid (< 2^31 nodes)
    int32_t sx, sy, sz;  // strides to the +x / +y / +z corner (0 where that corner is clamped)
    float fx, fy, fz;
    unsigned valid;      // bit (dz*4 + dy*2 + dx): corner inside the grid
};

__device__ __forceinline__ Cell3 make_cell3(const KParams &P, float ax, float ay, float az) {
    int ix, iy, iz;
    Cell3 c;
    cell(ax, P.nx, P.filter_weights, ix, c.fx);
    cell(ay, P.ny, P.filter_weights, iy, c.fy);
    cell(az, P.nz, P.filter_weights, iz, c.fz);
    const bool x0 = (unsigned)ix < (unsigned)P.nx, x1 = (unsigned)(ix + 1) < (unsigned)P.nx;
    const bool y0 = (unsigned)iy < (unsigned)P.ny, y1 = (unsigned)(iy + 1) < (unsigned)P.ny;
    const bool z0 = (unsigned)iz < (unsigned)P.nz, z1 = (unsigned)(iz + 1) < (unsigned)P.nz;
    // bit k = dz*4 + dy*2 + dx: per axis, the corners on each side form a fixed bit pattern
    const unsigned X = (x0 ? 0x55u : 0u) | (x1 ? 0xAAu : 0u);
    const unsigned Y = (y0 ? 0x33u : 0u) | (y1 ? 0xCCu : 0u);
    const unsigned Z = (z0 ? 0x0Fu : 0u) | (z1 ? 0xF0u : 0u);
    c.valid = X & Y & Z;
    const int cx = min(max(ix, 0), P.nx - 1), cy = min(max(iy, 0), P.ny - 1), cz = min(max(iz, 0), P.nz - 1);
    c.base = (cz * P.ny + cy) * P.nx + cx;
    c.sx = (x0 && x1) ? 1 : 0;
    c.sy = (y0 && y1) ? P.nx : 0;
    c.sz = (z0 && z1) ? P.nx * P.ny : 0;
    return c;
}

// Trilinear interpolation of the three wind components of one snapshot (border = 0).
template <typename W>
__device__ __forceinline__ void tri3(const void *slot, const Cell3 &c, float &ou, float &ov, float &ow) {
    float u[8], v[8], w[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        const int32_t idx = c.base + (dx ? c.sx : 0) + (dy ? c.sy : 0) + (dz ? c.sz : 0);
        u[k] = 0.f; v[k] = 0.f; w[k] = 0.f;
        if (c.valid & (1u << k)) Store<W>::load3(slot, idx, u[k], v[k], w[k]);
    }
    float a00 = lerp_(u[0], u[1], c.fx), a10 = lerp_(u[2], u[3], c.fx);
    float a01 = lerp_(u[4], u[5], c.fx), a11 = lerp_(u[6], u[7], c.fx);
    ou = lerp_(lerp_(a00, a10, c.fy), lerp_(a01, a11, c.fy), c.fz);
    a00 = lerp_(v[0], v[1], c.fx); a10 = lerp_(v[2], v[3], c.fx);
    a01 = lerp_(v[4], v[5], c.fx); a11 = lerp_(v[6], v[7], c.fx);
    ov = lerp_(lerp_(a00, a10, c.fy), lerp_(a01, a11, c.fy), c.fz);
    a00 = lerp_(w[0], w[1], c.fx); a10 = lerp_(w[2], w[3], c.fx);
    a01 = lerp_(w[4], w[5], c.fx); a11 = lerp_(w[6], w[7], c.fx);
    ow = lerp_(lerp_(a00, a10, c.fy), lerp_(a01, a11, c.fy), c.fz);
}

// Pair nodes of the last cell a particle sampled (window-pair layouts).  Consecutive samples of
// one particle (its RK4 stages, its next step) mostly fall in the same cell, whose nodes then
// need no new gathers; the values and the arithmetic are the same either way.  The cell is
// identified by its first corner's index in the padded pair buffer (`base`); 3D keeps 24 (back,
// front) float pairs (48 registers; 16-bit nodes converted when loaded; AdvBounds gives the
// launch shape), 2D 8 pairs (16 registers).
// Corner k + 1 of each x pair (k even) is kept as its difference from corner k, formed once when
// the cell is loaded: the x lerps of every later sample are then one paired FMA each, with the
// difference lerp2_ would form (same instruction, same rounding).
struct SampleCache {
    int32_t base;
    float2 c2d[2][4];  // 2D: (back, front) of u and v at corners 0, 2 and differences 1 - 0, 3 - 2
    float2 c2[3][8];   // 3D: (back, front) of u, v, w at even corners, differences at odd ones
    __device__ __forceinline__ void reset() { base = -1; }
};

// 3D window pair with a zero border (one node below, two above the grid on every axis): the
// coordinate is clamped to [-1, n], so every corner of the footprint is a node of the padded
// buffer and needs no validity test, and the footprint's first corner alone identifies the cell.
// Same values as make_cell3 + border addressing: inside [-1, n] the cell and fraction are
// identical; outside it every corner the original reads is outside the grid (0), and here the
// fraction is 0 with the weighted-away corner finite, so the interpolation is +0 either way.
// Padded node count of a window-pair buffer: (nx + 3) (ny + 3) (nz + 3) in 3D, (nx + 3) (ny + 3)
// in 2D.
#ifndef __CUDACC_RTC__
inline int64_t padded_pair_nodes(int dim, int64_t nx, int64_t ny, int64_t nz) {
    return (nx + 3) * (ny + 3) * (dim == 3 ? nz + 3 : 1);
}
#endif

struct PCell {
    int32_t base;        // padded node index of corner (ix, iy, iz)
    float fx, fy, fz;
};

// Cell of a padded-axis coordinate without the conversion unit.  a is clamped to [-1, n]
// (n < 2^22); a + 1.5 * 2^23 rounded toward -infinity lies in [2^23, 2^24), where the floats
// are the integers, so it is floor(a) + 1.5 * 2^23 exactly and its bit pattern is
// PCELL_BITS + floor(a).  The fraction a + (1.5 * 2^23 - t) equals a - floorf(a) bit for bit,
// the sign of a zero fraction included (an exact integer is subtracted either way).
constexpr uint32_t PCELL_BITS = 0x4B400000u;   // bit pattern of 1.5 * 2^23
__device__ __forceinline__ uint32_t pcell1(float a, float n, int fw, float &f) {
    a = fminf(fmaxf(a, -1.0f), n);
    const float t = __fadd_rd(a, 12582912.0f);
    f = a + (12582912.0f - t);
    if (fw) f = floorf(f * 256.0f + 0.5f) * (1.0f / 256.0f);
    return __float_as_uint(t);   // PCELL_BITS + floor(a)
}

// fw: the launch's filter_weights (0 where the variant has it off at compile time).  The
// index (iz + 1) pnxy + (iy + 1) pnx + (ix + 1) is formed from the bit patterns of pcell1 in
// wrapping 32-bit arithmetic, with the patterns' offset removed by one loop-invariant term.
__device__ __forceinline__ PCell make_pcell(const KParams &P, float ax, float ay, float az, int fw) {
    PCell c;
    const uint32_t bx = pcell1(ax, P.fn[0], fw, c.fx);
    const uint32_t by = pcell1(ay, P.fn[1], fw, c.fy);
    const uint32_t bz = pcell1(az, P.fn[2], fw, c.fz);
    const uint32_t sy = (uint32_t)P.pnx, sz = (uint32_t)P.pnxy;
    c.base = (int32_t)(bz * sz + by * sy + bx - (PCELL_BITS - 1u) * (sz + sy + 1u));
    return c;
}

// lerp_ on a (back, front) pair with one weight, as paired float32 instructions: b - a is formed
// as fma(a, -1, b) (the product is exact, so it rounds like the subtraction), then fma(t, d, a);
// each half equals lerp_ on that half bit for bit.
__device__ __forceinline__ float2 lerp2_(float2 a, float2 b, float t) {
    const float2 d = __ffma2_rn(a, make_float2(-1.f, -1.f), b);
    return __ffma2_rn(make_float2(t, t), d, a);
}

// b - a of lerp2_, formed alone (the sample cache stores it for the x pairs).
__device__ __forceinline__ float2 diff2_(float2 a, float2 b) { return __ffma2_rn(a, make_float2(-1.f, -1.f), b); }

// Trilinear interpolation of 8 corner pairs (odd entries: differences, SampleCache): x, then y,
// then z (the order of tri3).
__device__ __forceinline__ float2 tri8p(const float2 (&c)[8], float fx, float fy, float fz) {
    const float2 tx = make_float2(fx, fx);
    const float2 a00 = __ffma2_rn(tx, c[1], c[0]), a10 = __ffma2_rn(tx, c[3], c[2]);
    const float2 a01 = __ffma2_rn(tx, c[5], c[4]), a11 = __ffma2_rn(tx, c[7], c[6]);
    return lerp2_(lerp2_(a00, a10, fy), lerp2_(a01, a11, fy), fz);
}

// Loads the 8 padded corners of the cell at `base` into the sample cache as 24 (back, front)
// float pairs (u, v, w per corner); 16-bit nodes are converted once here, not per sample.
template <typename H>
__device__ __forceinline__ void fill_padded(const KParams &P, const void *pairs, int32_t base, SampleCache &cc) {
    const int32_t sy = P.pnx, sz = P.pnxy;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int32_t idx = base + ((k & 1) ? 1 : 0) + ((k & 2) ? sy : 0) + ((k & 4) ? sz : 0);
        float2 c[3];
        if constexpr (std::is_same<H, float>::value) {
            Store<Pair<float>>::load3p(pairs, idx, c);
        } else {
            const uint4 q = __ldg(reinterpret_cast<const uint4 *>(pairs) + idx);
            c[0] = Store<Pair<H>>::cvt(q.x);
            c[1] = Store<Pair<H>>::cvt(q.y);
            c[2] = Store<Pair<H>>::cvt(q.z);
        }
        if (k & 1) {
            cc.c2[0][k] = diff2_(cc.c2[0][k - 1], c[0]);
            cc.c2[1][k] = diff2_(cc.c2[1][k - 1], c[1]);
            cc.c2[2][k] = diff2_(cc.c2[2][k - 1], c[2]);
        } else {
            cc.c2[0][k] = c[0]; cc.c2[1][k] = c[1]; cc.c2[2][k] = c[2];
        }
    }
    cc.base = base;
}

// The cached corner pairs, reloaded when the cell changes; out[c] = (back, front) value of
// component c at the sample.  H: the pair's element type (float, bf16 or fp16).
template <typename H>
__device__ __forceinline__ void tri3p_padded(const KParams &P, const void *pairs, const PCell &c, SampleCache &cc,
                                             float2 (&out)[3]) {
    if (c.base != cc.base) fill_padded<H>(P, pairs, c.base, cc);
    out[0] = tri8p(cc.c2[0], c.fx, c.fy, c.fz);
    out[1] = tri8p(cc.c2[1], c.fx, c.fy, c.fz);
    out[2] = tri8p(cc.c2[2], c.fx, c.fy, c.fz);
}

template <typename W> struct PairElem { using type = void; };
template <typename H> struct PairElem<Pair<H>> { using type = H; };

// Trilinear interpolation of one scalar float32 plane.
__device__ __forceinline__ float tri1(const float *plane, const Cell3 &c) {
    float s[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int dx = k & 1, dy = (k >> 1) & 1, dz = (k >> 2) & 1;
        const int32_t idx = c.base + (dx ? c.sx : 0) + (dy ? c.sy : 0) + (dz ? c.sz : 0);
        s[k] = (c.valid & (1u << k)) ? __ldg(plane + idx) : 0.f;
    }
    const float a00 = lerp_(s[0], s[1], c.fx), a10 = lerp_(s[2], s[3], c.fx);
    const float a01 = lerp_(s[4], s[5], c.fx), a11 = lerp_(s[6], s[7], c.fx);
    return lerp_(lerp_(a00, a10, c.fy), lerp_(a01, a11, c.fy), c.fz);
}

// Bilinear footprint with clamped indices (2D pitch textures sample as clamp).
struct Cell2 {
    int32_t i00, i10, i01, i11;
    float fx, fy;
};

__device__ __forceinline__ Cell2 make_cell2(int nx, int ny, int fw, float ax, float ay) {
    int ix, iy;
    Cell2 c;
    cell(ax, nx, fw, ix, c.fx);
    cell(ay, ny, fw, iy, c.fy);
    const int x0 = min(max(ix, 0), nx - 1), x1 = min(max(ix + 1, 0), nx - 1);
    const int y0 = min(max(iy, 0), ny - 1), y1 = min(max(iy + 1, 0), ny - 1);
    c.i00 = y0 * nx + x0;
    c.i10 = y0 * nx + x1;
    c.i01 = y1 * nx + x0;
    c.i11 = y1 * nx + x1;
    return c;
}

template <typename W>
__device__ __forceinline__ void bil2(const void *slot, const Cell2 &c, float &ou, float &ov) {
    float u0, v0, u1, v1, u2, v2, u3, v3;
    Store<W>::load2(slot, c.i00, u0, v0);
    Store<W>::load2(slot, c.i10, u1, v1);
    Store<W>::load2(slot, c.i01, u2, v2);
    Store<W>::load2(slot, c.i11, u3, v3);
    ou = lerp_(lerp_(u0, u1, c.fx), lerp_(u2, u3, c.fx), c.fy);
    ov = lerp_(lerp_(v0, v1, c.fx), lerp_(v2, v3, c.fx), c.fy);
}

// 2D window pair with replicated edges: padded node (x, y), x in [-1, nx + 1] and y in
// [-1, ny + 1], of a (nx + 3) x (ny + 3) buffer holds node (clamp(x), clamp(y)), so a coordinate
// clamped to [-1, n] reads the clamp-addressed corners of make_cell2 without index clamps.  Same
// values: inside [-1, n] cell, fraction and corners are unchanged; outside it both corners of the
// axis are the same edge node, interpolated with any fraction to that node's value exactly.
// The cache keeps the 4 corners as floats (16 registers), keyed by the first corner's index.
template <typename W>
__device__ __forceinline__ void bil2p_padded(const KParams &P, const void *pairs, float ax, float ay, int fw,
                                             SampleCache &cc, float2 (&out)[2]) {
    float fx, fy;
    const uint32_t bx = pcell1(ax, P.fn[0], fw, fx);
    const uint32_t by = pcell1(ay, P.fn[1], fw, fy);
    const uint32_t sy = (uint32_t)P.pnx;
    const int32_t base = (int32_t)(by * sy + bx - (PCELL_BITS - 1u) * (sy + 1u));   // (iy + 1) pnx + (ix + 1)
    if (base != cc.base) {
        const int32_t idx[4] = {base, base + 1, base + P.pnx, base + P.pnx + 1};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float2 c[2];
            Store<W>::load2p(pairs, idx[k], c);
            cc.c2d[0][k] = (k & 1) ? diff2_(cc.c2d[0][k - 1], c[0]) : c[0];
            cc.c2d[1][k] = (k & 1) ? diff2_(cc.c2d[1][k - 1], c[1]) : c[1];
        }
        cc.base = base;
    }
#pragma unroll
    for (int k = 0; k < 2; ++k)
        out[k] = lerp2_(__ffma2_rn(make_float2(fx, fx), cc.c2d[k][1], cc.c2d[k][0]),
                        __ffma2_rn(make_float2(fx, fx), cc.c2d[k][3], cc.c2d[k][2]), fy);
}


__device__ __forceinline__ float bil1(const float *plane, const Cell2 &c) {
    return lerp_(lerp_(__ldg(plane + c.i00), __ldg(plane + c.i10), c.fx),
                 lerp_(__ldg(plane + c.i01), __ldg(plane + c.i11), c.fx), c.fy);
}

struct V3 {
    float x, y, z;
};

__device__ __forceinline__ float dot3(const V3 &a, const V3 &b, int dim) {
    float s = a.x * b.x;
    s = __fmaf_rn(a.y, b.y, s);
    if (dim == 3) s = __fmaf_rn(a.z, b.z, s);
    return s;
}

// Wind at world position p, time weight t: interpolate() of TrajectoryIntegrator.icc:42-110.
// FT: the step kernel's feature set; lean variants run with filter_weights off (kernel_features).
template <int DIM, typename W, int FT = FT_GENERIC>
__device__ __forceinline__ V3 wind_at(const KParams &P, const V3 &p, float t, const void *wb, const void *wf,
                                      SampleCache &cc) {
    V3 r{0.f, 0.f, 0.f};
    const int fw = (FT & FT_LEAN) ? 0 : P.filter_weights;
    const float ax = (p.x - P.off[0]) * P.inv_scale[0];
    const float ay = (p.y - P.off[1]) * P.inv_scale[1];
    if constexpr (IsPair<W>::value) {
        // window-pair layout (dynamic wind only): wb points at the pair buffer
        if (DIM == 3) {
            const float az = (p.z - P.off[2]) * P.inv_scale[2];
            const PCell c = make_pcell(P, ax, ay, az, fw);
            float2 bf[3];
            using H = typename PairElem<W>::type;
            tri3p_padded<H>(P, wb, c, cc, bf);
            r.x = lerp_(bf[0].x, bf[0].y, t); r.y = lerp_(bf[1].x, bf[1].y, t); r.z = lerp_(bf[2].x, bf[2].y, t);
        } else {
            float2 bf[2];
            bil2p_padded<W>(P, wb, ax, ay, fw, cc, bf);
            r.x = lerp_(bf[0].x, bf[0].y, t); r.y = lerp_(bf[1].x, bf[1].y, t);
        }
        return r;
    } else {
    if (DIM == 3) {
        const float az = (p.z - P.off[2]) * P.inv_scale[2];
        const Cell3 c = make_cell3(P, ax, ay, az);
        float bu, bv, bw;
        tri3<W>(wb, c, bu, bv, bw);
        if (P.wind_dynamic) {
            float fu, fv, fw;
            tri3<W>(wf, c, fu, fv, fw);
            r.x = lerp_(bu, fu, t); r.y = lerp_(bv, fv, t); r.z = lerp_(bw, fw, t);
        } else {
            r.x = bu; r.y = bv; r.z = bw;
        }
    } else {
        const Cell2 c = make_cell2(P.nx, P.ny, P.filter_weights, ax, ay);
        float bu, bv;
        bil2<W>(wb, c, bu, bv);
        if (P.wind_dynamic) {
            float fu, fv;
            bil2<W>(wf, c, fu, fv);
            r.x = lerp_(bu, fu, t); r.y = lerp_(bv, fv, t);
        } else {
            r.x = bu; r.y = bv;
        }
    }
    return r;
    }
}

template <int DIM, typename W>
__device__ __forceinline__ V3 wind_at(const KParams &P, const V3 &p, float t, const void *wb, const void *wf) {
    SampleCache cc;
    cc.reset();
    return wind_at<DIM, W>(P, p, t, wb, wf, cc);
}

// sphere_coordinates (TrajectoryIntegrator.tpp:98-104).
__device__ __forceinline__ V3 sphere_(const KParams &P, float py, V3 v) {
    const float pi = 3.14159265358979323846f;
    V3 r{0.f, 0.f, 0.f};
    r.x = (v.x * 180.f) / (P.sphere_radius * cosf(py * (pi * 2.f) / 360.f) * pi);
    r.y = (v.y * 180.f) / (pi * P.sphere_radius);
    return r;
}

__device__ __forceinline__ float ref_at(const float (&ref)[19], int i) {
    switch (i) {
        case 0: return ref[0]; case 1: return ref[1]; case 2: return ref[2]; case 3: return ref[3];
        case 4: return ref[4]; case 5: return ref[5]; case 6: return ref[6]; case 7: return ref[7];
        case 8: return ref[8]; case 9: return ref[9]; case 10: return ref[10]; case 11: return ref[11];
        case 12: return ref[12]; case 13: return ref[13]; case 14: return ref[14]; case 15: return ref[15];
        case 16: return ref[16]; case 17: return ref[17]; default: return ref[18];
    }
}

// Expression programs in kernel parameter space (deferred_extras_kernel): read through the
// constant cache at a warp-uniform index, so the dispatch below branches on uniform values and
// no global load sits on the evaluation's critical path.  Programs longer in total than
// GR_EXPR_PARAM_CODE are read from global memory (KParams::prog) instead.
constexpr int GR_EXPR_PARAM_CODE = 512;
struct ExprSet {
    int32_t in_params;                 // 1: code[] holds the programs
    int32_t start[GR_MAX_EXPR], len[GR_MAX_EXPR];
    Instr code[GR_EXPR_PARAM_CODE];
};

// Program sources of eval_program: expression e's length and instruction k; eval(e, ref) is the
// value of expression e (the interpreter here, straight-line code in a run-time compiled JitCode).
struct GlobalCode {
    const Program *prog;
    __device__ __forceinline__ int len(int e) const { return prog[e].len; }
    __device__ __forceinline__ Instr at(int e, int k) const { return prog[e].code[k]; }
    __device__ __forceinline__ float eval(int e, const float (&ref)[19]) const;
};
struct ParamCode {
    const ExprSet &X;
    __device__ __forceinline__ int len(int e) const { return X.len[e]; }
    __device__ __forceinline__ Instr at(int e, int k) const { return X.code[X.start[e] + k]; }
    __device__ __forceinline__ float eval(int e, const float (&ref)[19]) const;
};

// Postfix evaluation with an 8-register rotating stack (s0 = top); the program is uniform
// across the grid, so every branch here is uniform.
template <typename Code>
__device__ __forceinline__ float eval_program(const Code &code, int e, const float (&ref)[19]) {
    float s0 = 0.f, s1 = 0.f, s2 = 0.f, s3 = 0.f, s4 = 0.f, s5 = 0.f, s6 = 0.f, s7 = 0.f;
    const int len = code.len(e);
    for (int k = 0; k < len; ++k) {
        const Instr in = code.at(e, k);
        float r;
        bool binary = false, push = false;
        switch (in.op) {
            case OP_REF: r = ref_at(ref, in.arg); push = true; break;
            case OP_CONST: r = in.value; push = true; break;
            case OP_ADD: r = s1 + s0; binary = true; break;
            case OP_SUB: r = s1 - s0; binary = true; break;
            case OP_MUL: r = s1 * s0; binary = true; break;
            case OP_DIV: r = s1 / s0; binary = true; break;
            case OP_RSUB: r = s0 - s1; binary = true; break;
            case OP_RDIV: r = s0 / s1; binary = true; break;
            case OP_ATAN2: r = atan2f(s1, s0); binary = true; break;
            case OP_RATAN2: r = atan2f(s0, s1); binary = true; break;
            case OP_SQRT: r = sqrtf(s0); break;
            case OP_EXP: r = expf(s0); break;
            case OP_LOG: r = logf(s0); break;
            case OP_SIN: r = sinf(s0); break;
            case OP_COS: r = cosf(s0); break;
            case OP_TAN: r = tanf(s0); break;
            case OP_ASIN: r = asinf(s0); break;
            case OP_ACOS: r = acosf(s0); break;
            case OP_ATAN: r = atanf(s0); break;
            default: r = s0; break;
        }
        if (push) {
            s7 = s6; s6 = s5; s5 = s4; s4 = s3; s3 = s2; s2 = s1; s1 = s0; s0 = r;
        } else if (binary) {
            s0 = r; s1 = s2; s2 = s3; s3 = s4; s4 = s5; s5 = s6; s6 = s7;
        } else {
            s0 = r;
        }
    }
    return s0;
}

__device__ __forceinline__ float GlobalCode::eval(int e, const float (&ref)[19]) const { return eval_program(*this, e, ref); }
__device__ __forceinline__ float ParamCode::eval(int e, const float (&ref)[19]) const { return eval_program(*this, e, ref); }

// The run's volume / expression options as the code below reads them: the KParams fields, or
// compile-time constants in the run-time compiled deferred kernel (jit.cu defines
// GR_JIT_OPTIONS and GR_JIT_<field>), where the loops and branches a run does not use drop out.
#ifdef GR_JIT_OPTIONS
#define GR_OPT(P, name) (GR_JIT_##name)
#else
#define GR_OPT(P, name) ((P).name)
#endif

// Volume samples and expression values of a particle, evaluated from the inputs of its last
// alive step: position p (that step's new position), stage-averaged velocity vc, curvature cv
// and the step's time weight / ring slots (tpp:363-447).  The kernel calls this only when the
// values become observable (a record, the end of a launch), which gives the same values as
// evaluating after every alive step, as the reference does.
template <int DIM, typename Code>
__device__ __forceinline__ void eval_extras(const KParams &P, const Code &code, const StepEntry &E, int64_t pid,
                                            const V3 &p, const V3 &vc, float cv, float (&vol)[GR_MAX_VOL],
                                            float (&cmp)[GR_MAX_EXPR]) {
    const float t0 = GR_OPT(P, dyn_any) ? E.t0 : 0.f;
    if (GR_OPT(P, volume_mode) != 0 && GR_OPT(P, nvol) > 0) {
        const int vb = GR_OPT(P, volume_mode) == 2 ? E.slot_back : 0, vf = GR_OPT(P, volume_mode) == 2 ? E.slot_front : 0;
        const float ax = (p.x - P.off[0]) * P.inv_scale[0];
        const float ay = (p.y - P.off[1]) * P.inv_scale[1];
        if (DIM == 3) {
            const float az = (p.z - P.off[2]) * P.inv_scale[2];
            const Cell3 c = make_cell3(P, ax, ay, az);
#pragma unroll
            for (int k = 0; k < GR_MAX_VOL; ++k) {
                if (k < GR_OPT(P, nvol)) {
                    const float b = tri1(P.vol + ((int64_t)vb * GR_MAX_VOL + k) * P.vol_plane, c);
                    vol[k] = GR_OPT(P, volume_mode) == 2 ? lerp_(b, tri1(P.vol + ((int64_t)vf * GR_MAX_VOL + k) * P.vol_plane, c), t0)
                                                : b;
                }
            }
        } else {
            const Cell2 c = make_cell2(P.nx, P.ny, P.filter_weights, ax, ay);
#pragma unroll
            for (int k = 0; k < GR_MAX_VOL; ++k) {
                if (k < GR_OPT(P, nvol)) {
                    const float b = bil1(P.vol + ((int64_t)vb * GR_MAX_VOL + k) * P.vol_plane, c);
                    vol[k] = GR_OPT(P, volume_mode) == 2 ? lerp_(b, bil1(P.vol + ((int64_t)vf * GR_MAX_VOL + k) * P.vol_plane, c), t0)
                                                : b;
                }
            }
        }
    }
    if (GR_OPT(P, nexpr) > 0) {
        float ref[19];
        ref[0] = p.x; ref[1] = p.y; ref[2] = DIM == 3 ? p.z : 0.f;
        ref[3] = GR_OPT(P, curvature_mode) == 3 ? cv : 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) ref[4 + k] = k < GR_OPT(P, nvol) ? vol[k] : 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float c = 0.f;
            if (k < GR_OPT(P, ncon) && GR_OPT(P, constants_mode) != 0) {
                const int cb = GR_OPT(P, constants_mode) == 2 ? E.slot_back : 0;
                const float b = __ldg(P.cons + ((int64_t)cb * GR_MAX_CON + k) * P.n_total + pid);
                if (GR_OPT(P, constants_mode) == 2) {
                    const float f = __ldg(P.cons + ((int64_t)E.slot_front * GR_MAX_CON + k) * P.n_total + pid);
                    c = lerp_(b, f, t0);
                } else {
                    c = b;
                }
            }
            ref[12 + k] = c;
        }
        ref[16] = vc.x; ref[17] = vc.y; ref[18] = DIM == 3 ? vc.z : 0.f;
#pragma unroll
        for (int e = 0; e < GR_MAX_EXPR; ++e)
            if (e < GR_OPT(P, nexpr)) cmp[e] = code.eval(e, ref);
    }
}

// The volume / expression values of slot i kept in the state arrays between evaluations.  For
// an evaluation (`evaluating`) only what eval_extras reads but does not overwrite is loaded:
// volumes when no volume is sampled (their stored values enter the expressions).
__device__ __forceinline__ void load_extras(const KParams &P, int64_t i, bool evaluating, float (&vol)[GR_MAX_VOL],
                                            float (&cmp)[GR_MAX_EXPR]) {
    const bool vols = !evaluating || GR_OPT(P, volume_mode) == 0;
#pragma unroll
    for (int k = 0; k < GR_MAX_VOL; ++k) vol[k] = (k < GR_OPT(P, nvol) && vols) ? P.volc[k * P.n_state + i] : 0.f;
#pragma unroll
    for (int k = 0; k < GR_MAX_EXPR; ++k) cmp[k] = (k < GR_OPT(P, nexpr) && !evaluating) ? P.cmpc[k * P.n_state + i] : 0.f;
}

__device__ __forceinline__ void store_extras(const KParams &P, int64_t i, const float (&vol)[GR_MAX_VOL],
                                             const float (&cmp)[GR_MAX_EXPR]) {
#pragma unroll
    for (int k = 0; k < GR_MAX_VOL; ++k)
        if (k < GR_OPT(P, nvol)) P.volc[k * P.n_state + i] = vol[k];
#pragma unroll
    for (int k = 0; k < GR_MAX_EXPR; ++k)
        if (k < GR_OPT(P, nexpr)) P.cmpc[k * P.n_state + i] = cmp[k];
}

// ------------------------------------------------------------------ the step kernel

// Volume / expression values at a record or at the end of a launch (tpp:363-435): evaluated if
// an alive step has passed since the last evaluation (`dirty`, then kept in the state arrays),
// else the state arrays' values; written to the record's rows when irec >= 0.
template <int DIM, typename Code>
__device__ __forceinline__ void extras_at(const KParams &P, const Code &code, int64_t i, int64_t pid, bool dirty,
                                          int last_s, const V3 &p, const V3 &vc_last, float cv, int32_t irec) {
    float vol[GR_MAX_VOL], cmp[GR_MAX_EXPR];
    load_extras(P, i, dirty, vol, cmp);
    if (dirty) {
        eval_extras<DIM>(P, code, P.sched[last_s], pid, p, vc_last, cv, vol, cmp);
        store_extras(P, i, vol, cmp);
    }
    if (irec < 0) return;
    if (GR_OPT(P, volume_mode) != 0) {
#pragma unroll
        for (int k = 0; k < GR_MAX_VOL; ++k)
            if (k < GR_OPT(P, nvol)) P.hvol[((int64_t)k * P.Li + irec) * P.n_total + pid] = vol[k];
    }
#pragma unroll
    for (int e = 0; e < GR_MAX_EXPR; ++e)
        if (e < GR_OPT(P, nexpr)) P.hcmp[((int64_t)e * P.Li + irec) * P.n_total + pid] = cmp[e];
}

// extras_at for the step kernel's in-kernel evaluation (FT_EXTRAS).  Not inlined: it runs once
// per record, and its register peak (the expression stack, the volume samples) then stays out
// of the step loop's allocation; the caller's live registers are saved around the call.
template <int DIM>
__device__ __noinline__ void record_extras(const KParams &P, int64_t i, int64_t pid, bool dirty, int last_s,
                                           V3 p, V3 vc_last, float cv, int32_t irec) {
    extras_at<DIM>(P, GlobalCode{P.prog}, i, pid, dirty, last_s, p, vc_last, cv, irec);
}

// Volume / expression values after a FT_DEFER step launch (tpp:363-435), from the inputs of a
// slot's last moved step: its position (a particle keeps it once it stops), the stored
// velocity and that step's schedule entry.  Same values as the in-kernel evaluation.
//  - rec >= 0: the launch saved record rec (info record irec) at one step: every slot of the live
//    prefix writes the record's rows, evaluating first if it moved since its last evaluation
//    (inputs and position in vrec, as of the save step).
//  - rec < 0: slots with pending inputs (vlast) are evaluated into the state arrays: all of them
//    (all = 1, the end of a run) or those about to retire (aborted, or lifetime over by k_end),
//    whose values are final.  (Folding this pass into the record kernel measured slower: the
//    second evaluation path doubles the kernel's code.)
template <int DIM, typename Code>
__device__ __forceinline__ void deferred_extras(const KParams &P, const Code &code, int32_t rec, int32_t irec,
                                                int32_t k_end, int32_t all) {
    const int64_t n = P.n_dev ? (int64_t)*P.n_dev : P.n;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        if (rec >= 0) {
            const int64_t pid = P.id[i];
            const float cv = GR_OPT(P, curvature_mode) == 3 ? P.curv[i] : 0.f;
            const float4 a = P.vrec[2 * i], v = P.vrec[2 * i + 1];
            const int32_t last_s = __float_as_int(v.w);
            extras_at<DIM>(P, code, i, pid, last_s >= 0, last_s < 0 ? 0 : last_s, V3{a.x, a.y, a.z},
                           V3{v.x, v.y, v.z}, cv, irec);
        } else {
            if (!all && P.status[i] == 0 && !(P.life && P.life[i] <= k_end)) continue;
            const float4 v = P.vlast[i];
            const int32_t last_s = __float_as_int(v.w);
            if (last_s < 0) continue;
            const int64_t pid = P.id[i];
            const float cv = GR_OPT(P, curvature_mode) == 3 ? P.curv[i] : 0.f;
            const V3 p{P.px[i], P.py[i], DIM == 3 ? P.pz[i] : 0.f};
            extras_at<DIM>(P, code, i, pid, true, last_s, p, V3{v.x, v.y, v.z}, cv, -1);
            reinterpret_cast<int32_t *>(P.vlast + i)[3] = -1;
        }
    }
}

template <int DIM>
__global__ void __launch_bounds__(256, 3) deferred_extras_kernel(const __grid_constant__ KParams P,
                                                              const __grid_constant__ ExprSet X, int32_t rec,
                                                              int32_t irec, int32_t k_end, int32_t all) {
    if (X.in_params)
        deferred_extras<DIM>(P, ParamCode{X}, rec, irec, k_end, all);
    else
        deferred_extras<DIM>(P, GlobalCode{P.prog}, rec, irec, k_end, all);
}

#ifndef GR_ADV_MIN_BLOCKS
#define GR_ADV_MIN_BLOCKS 2
#endif

// Advances the particle in slot i through steps [s0, s1) (or until its lifetime ends).
template <int DIM, bool RK4, typename W, int FT>
__device__ __forceinline__ void advance_particle(const KParams &P, const int64_t i, const int64_t n_live,
                                                 unsigned long long &steps_acc, unsigned &alive_acc) {
    // options: runtime values in the generic variant; in a lean variant (FT_LEAN) the ones the
    // host checked are off, and curvature / extras are the variant's compile-time choice
    constexpr bool LEAN = (FT & FT_LEAN) != 0;
    const int curvature_mode = LEAN ? ((FT & FT_CURV) ? 1 : 0) : P.curvature_mode;
    const int abort_mode = LEAN ? 0 : P.abort_mode;
    const int uplift_mode = LEAN ? 0 : P.uplift_mode;
    const bool compensated = LEAN ? (FT & FT_COMP) != 0 : P.compensated != 0;
    const bool topography = LEAN ? false : P.topography != 0;
    const int border_mode = LEAN ? 0 : P.border_mode;
    unsigned *const alive_at = LEAN ? nullptr : P.alive_at;
    const bool valid = i < n_live;
    int32_t st = valid ? P.status[i] : 1;
    bool alive = st == 0;
    const int64_t pid = valid ? (int64_t)P.id[i] : 0;

    V3 p{0.f, 0.f, 0.f}, q{0.f, 0.f, 0.f}, comp{0.f, 0.f, 0.f}, ld{0.f, 0.f, 0.f};
    float len = 0.f, tc = 0.f, cv = 0.f;

    const bool curv_prev = curvature_mode == 1 || curvature_mode == 3;
    float seg = 0.f;   // |p - q| (curvature's ds): carried from the step that formed it
    if (valid) {
        p.x = P.px[i]; p.y = P.py[i];
        if (DIM == 3) p.z = P.pz[i];
        if (curv_prev) {
            q.x = P.qx[i]; q.y = P.qy[i]; if (DIM == 3) q.z = P.qz[i];
            const V3 a{p.x - q.x, p.y - q.y, p.z - q.z};
            seg = sqrtf(dot3(a, a, DIM));
        }
        if (compensated) { comp.x = P.kx[i]; comp.y = P.ky[i]; if (DIM == 3) comp.z = P.kz[i]; }
        if (curvature_mode == 2) { ld.x = P.lx[i]; ld.y = P.ly[i]; if (DIM == 3) ld.z = P.lz[i]; }
        if (abort_mode != 0) len = P.length[i];
        if (curvature_mode != 0) tc = P.tc[i];
        if (curvature_mode == 3) cv = P.curv[i];
    }
    const bool was_alive = alive;
    unsigned long long my_steps = 0;
    const int32_t life = (valid && P.life) ? P.life[i] : 0x7fffffff;   // steps this particle may run
    const int32_t birth = (valid && P.birth) ? P.birth[i] : 0;          // first step it runs
    const bool extras = LEAN ? (FT & FT_EXTRAS) != 0 : ((P.volume_mode != 0 && P.nvol > 0) || P.nexpr > 0);
    V3 vc_last{0.f, 0.f, 0.f};
    int last_s = P.s0;
    bool dirty = false;   // volumes / expressions not yet evaluated for the last alive step
    const int sph = !LEAN && P.sphere && DIM == 2;

    SampleCache cc;
    cc.reset();
    for (int s = P.s0; s < P.s1; ++s) {
        const StepEntry E = P.sched[s];
        if (alive && s < life && s >= birth) {
            ++my_steps;
            const int sb = P.wind_dynamic ? E.slot_back : 0, sf = P.wind_dynamic ? E.slot_front : 0;
            const void *wb = IsPair<W>::value ? P.pair : reinterpret_cast<const char *>(P.wind) + (int64_t)sb * P.wind_stride;
            const void *wf = reinterpret_cast<const char *>(P.wind) + (int64_t)sf * P.wind_stride;
            const float t0 = P.dyn_any ? E.t0 : 0.f;

            // integrator (tpp:135-231)
            V3 v, vc;
            if (RK4) {
                // the four stages as one loop (one copy of the sampling code, which keeps the
                // step loop within the instruction cache): stage k samples at a with its time
                // weight, and the sum ((k1 + 2 k2) + 2 k3) + k4 is accumulated in that order
                V3 a = p, acc{0.f, 0.f, 0.f}, accc{0.f, 0.f, 0.f};
#pragma unroll 1
                for (int stage = 0; stage < 4; ++stage) {
                    const float tw = stage == 0 ? t0 : (stage == 3 ? E.t2 : E.t1);
                    const V3 kc = wind_at<DIM, W, FT>(P, a, tw, wb, wf, cc);
                    const V3 k = sph ? sphere_(P, a.y, kc) : kc;
                    if (stage == 0) {
                        acc = k;
                        accc = kc;
                    } else {
                        const float wgt = stage == 3 ? 1.f : 2.f;   // 1 * k is exact: the same sum
                        acc = V3{acc.x + wgt * k.x, acc.y + wgt * k.y, acc.z + wgt * k.z};
                        if (sph) accc = V3{accc.x + wgt * kc.x, accc.y + wgt * kc.y, 0.f};
                    }
                    const float c = stage < 2 ? P.hh : P.h;
                    a = V3{__fmaf_rn(k.x, c, p.x), __fmaf_rn(k.y, c, p.y), DIM == 3 ? __fmaf_rn(k.z, c, p.z) : 0.f};
                }
                v.x = acc.x * P.sixth;
                v.y = acc.y * P.sixth;
                v.z = DIM == 3 ? acc.z * P.sixth : 0.f;
                if (sph) {
                    vc.x = accc.x * P.sixth;
                    vc.y = accc.y * P.sixth;
                    vc.z = 0.f;
                } else {
                    vc = v;
                }
            } else {
                vc = wind_at<DIM, W, FT>(P, p, t0, wb, wf, cc);
                v = sph ? sphere_(P, p.y, vc) : vc;
            }

            // displacement, reverse and uplift (tpp:233-250)
            V3 dp{v.x * P.h, v.y * P.h, DIM == 3 ? v.z * P.h : 0.f};
            if (P.reverse) { dp.x = -dp.x; dp.y = -dp.y; dp.z = -dp.z; }
            if (DIM == 3 && uplift_mode != 0) {
                const int lb = uplift_mode == 2 ? E.slot_back : 0, lf = uplift_mode == 2 ? E.slot_front : 0;
                const float *LB = P.lift + (int64_t)lb * P.n_total * 3 + pid * 3;
                const float *LF = P.lift + (int64_t)lf * P.n_total * 3 + pid * 3;
                if (uplift_mode == 1) {
                    dp.x = dp.x + LB[0]; dp.y = dp.y + LB[1]; dp.z = dp.z + LB[2];
                } else {
                    dp.x = dp.x + lerp_(LB[0], LF[0], t0);
                    dp.y = dp.y + lerp_(LB[1], LF[1], t0);
                    dp.z = dp.z + lerp_(LB[2], LF[2], t0);
                }
            }

            // length abort (tpp:252-280)
            int32_t abort = 0;
            if (abort_mode != 0) {
                const float dpl = sqrtf(dot3(dp, dp, DIM));
                const float nl = len + dpl;
                if (abort_mode == 2) {
                    if (nl > P.max_length) {
                        const float sc = (P.max_length - len) / dpl;
                        dp.x = sc * dp.x; dp.y = sc * dp.y; dp.z = sc * dp.z;
                        len = P.max_length;
                        abort = 1;
                    } else {
                        len = nl;
                    }
                } else {
                    if (nl > P.max_length) abort = 1;
                    len = nl;
                }
            }

            // new position (tpp:282); Kahan-compensated in the precision form
            V3 np;
            if (compensated) {
                const V3 sd{P.reverse ? -dp.x : dp.x, P.reverse ? -dp.y : dp.y, P.reverse ? -dp.z : dp.z};
                float y = sd.x - comp.x, t = p.x + y;
                np.x = t; comp.x = (t - p.x) - y;
                y = sd.y - comp.y; t = p.y + y;
                np.y = t; comp.y = (t - p.y) - y;
                if (DIM == 3) { y = sd.z - comp.z; t = p.z + y; np.z = t; comp.z = (t - p.z) - y; }
                else np.z = 0.f;
            } else {
                np.x = P.reverse ? p.x - dp.x : p.x + dp.x;
                np.y = P.reverse ? p.y - dp.y : p.y + dp.y;
                np.z = DIM == 3 ? (P.reverse ? p.z - dp.z : p.z + dp.z) : 0.f;
            }

            // border and abort checks (tpp:284-323, icc:7-20, tpp:13-96)
            if (abort == 0) {
                const float dp2 = dot3(dp, dp, DIM);
                const int bm = DIM == 3 ? 0 : border_mode;
                if (bm == 0) {
                    bool topo = false;
                    if (DIM == 3 && topography) {
                        const Cell2 c = make_cell2(P.nx, P.ny, P.filter_weights, np.x / P.scale[0], np.y / P.scale[1]);
                        topo = bil1(P.topo, c) > np.z;
                    }
                    if (topo) abort = 3;
                    else if (dp2 < 1e-9f) abort = 4;
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
            }

            st = abort;
            if (abort == 2 || abort == 3 || abort == 4) {
                // old position kept, total curvature flagged (tpp:327-332)
                if (curvature_mode != 0) tc = -1.f;
                alive = false;
            } else {
                // curvature (tpp:335-361)
                if (curvature_mode == 2) {
                    const float inv = 1.0f / sqrtf(dot3(v, v, DIM));
                    const V3 u{v.x * inv, v.y * inv, v.z * inv};
                    if (E.flags & SF_TIME_POS) {
                        const float k = acosf(dot3(ld, u, DIM));
                        if (!isnan(k)) tc += k;
                    }
                    ld = u;
                } else if (curv_prev) {
                    // |np - p|: this segment's length, the next step's |p - q|
                    const V3 b{np.x - p.x, np.y - p.y, np.z - p.z};
                    const float nseg = sqrtf(dot3(b, b, DIM));
                    if (E.flags & SF_TIME_POS) {
                        float k = 0.f;
                        if (DIM == 3) {
                            // central differences scaled by the float reciprocals of 2 h and h h
                            // (the reference divides, icc:151-154: within one rounding of these)
                            const V3 d1{(np.x - q.x) * P.inv_2h, (np.y - q.y) * P.inv_2h, (np.z - q.z) * P.inv_2h};
                            const V3 d2{((q.x + np.x) - 2.f * p.x) * P.inv_hh, ((q.y + np.y) - 2.f * p.y) * P.inv_hh,
                                        ((q.z + np.z) - 2.f * p.z) * P.inv_hh};
                            const V3 x{d1.y * d2.z - d1.z * d2.y, d1.z * d2.x - d1.x * d2.z, d1.x * d2.y - d1.y * d2.x};
                            const float l = sqrtf(dot3(d1, d1, 3));
                            k = fabsf(sqrtf(dot3(x, x, 3)) / (l * l * l));
                        }
                        const float ds = 0.5f * (seg + nseg);
                        if (curvature_mode == 3) cv = k;
                        if (!isnan(k)) tc += k * ds;
                    }
                    seg = nseg;
                }

                // volumes and expressions are evaluated lazily (eval_extras), or after the launch
                // from the stored inputs (FT_DEFER, deferred_extras_kernel)
                if constexpr ((FT & FT_DEFER) != 0)
                    P.vlast[i] = make_float4(vc.x, vc.y, DIM == 3 ? vc.z : 0.f, __int_as_float(s));
                vc_last = vc;
                last_s = s;
                dirty = true;

                q = p;
                p = np;
                if (abort != 0) alive = false;
            }
        }

        if (valid && (E.flags & SF_SAVE)) {
            float *hp = P.hpos + ((int64_t)E.rec * P.n_total + pid) * DIM;
            hp[0] = p.x; hp[1] = p.y;
            if (DIM == 3) hp[2] = p.z;
            if (curvature_mode == 3 && (E.flags & SF_CURV_REC)) P.hcurv[(int64_t)E.crec * P.n_total + pid] = cv;
            if constexpr ((FT & FT_DEFER) != 0) {
                // the record's inputs: the position and the last moved step's (if any since the
                // last evaluation)
                const float4 v = P.vlast[i];
                P.vrec[2 * i] = make_float4(p.x, p.y, DIM == 3 ? p.z : 0.f, 0.f);
                P.vrec[2 * i + 1] = v;
                if (__float_as_int(v.w) >= 0) reinterpret_cast<int32_t *>(P.vlast + i)[3] = -1;
            }
            if (extras) {
                record_extras<DIM>(P, i, pid, dirty, last_s, p, vc_last, cv, E.irec);
                dirty = false;
                // refill the sample cache for the next step's first sample (at p): the cached
                // nodes are then dead while the values above are evaluated, which frees their
                // registers there
                if constexpr (IsPair<W>::value && DIM == 3) {
                    const PCell c = make_pcell(P, (p.x - P.off[0]) * P.inv_scale[0], (p.y - P.off[1]) * P.inv_scale[1],
                                               (p.z - P.off[2]) * P.inv_scale[2], LEAN ? 0 : P.filter_weights);
                    fill_padded<typename PairElem<W>::type>(P, P.pair, c.base, cc);
                }
            }
        }

        // MinimumAliveParticles: particles alive after this step, one atomic per warp, spread
        // over 32 counters so that one address does not serialise the warps of the grid
        if (alive_at) {
            const unsigned m = __ballot_sync(0xffffffffu, valid && alive);
            if ((threadIdx.x & 31) == 0 && m)
                atomicAdd(alive_at + (int64_t)(s - P.s0) * 32 + (blockIdx.x & 31), (unsigned)__popc(m));
        }
    }

    if (valid && was_alive) {
        if (extras && dirty) record_extras<DIM>(P, i, pid, true, last_s, p, vc_last, cv, -1);
        P.status[i] = st;
        P.px[i] = p.x; P.py[i] = p.y;
        if (DIM == 3) P.pz[i] = p.z;
        if (curv_prev) { P.qx[i] = q.x; P.qy[i] = q.y; if (DIM == 3) P.qz[i] = q.z; }
        if (compensated) { P.kx[i] = comp.x; P.ky[i] = comp.y; if (DIM == 3) P.kz[i] = comp.z; }
        if (curvature_mode == 2) { P.lx[i] = ld.x; P.ly[i] = ld.y; if (DIM == 3) P.lz[i] = ld.z; }
        if (abort_mode != 0) P.length[i] = len;
        if (curvature_mode != 0) P.tc[i] = tc;
        if (curvature_mode == 3) P.curv[i] = cv;
    }

    steps_acc += my_steps;
    alive_acc += (valid && alive) ? 1u : 0u;
}

// One thread per particle, or (P.grid_stride) a persistent grid striding over the live
// prefix, whose size is read on the device: the launch shape then stays fixed while the live
// count shrinks, as a captured CUDA graph needs.
// Launch bounds: 256 threads, 2 blocks per SM (128 registers).  The float32 3D pair kernel keeps
// 48 cached floats in 128-thread blocks: 4 per SM (128 registers) in the generic variant and the
// lean ones with volume / expression values or with both Kahan positions and curvature, 5 per SM
// (96 registers, 20 warps) in the other lean ones, whose state fits there without spills; the
// extra warps hide more of the sampling and curvature latency.  The 16-bit kernels: AdvBounds16.
template <int DIM, typename W, int FT> struct AdvBounds { static constexpr int threads = 256, blocks = GR_ADV_MIN_BLOCKS; };
#ifndef GR_F32_PAIR_BLOCKS
#define GR_F32_PAIR_BLOCKS 4
#endif
#ifndef GR_F32_LIGHT_BLOCKS
#define GR_F32_LIGHT_BLOCKS 5
#endif
// 16-bit 3D pair kernels: 128 x 5 for the lean variants with curvature or deferred values
// (measured 5-6% faster than 256 x 2 on the 3D benchmark configuration), 256 x 2 for the rest
// (the positions-only variant of the batching and serving forms measured 2% slower at 128 x 5).
template <typename H, int FT> struct AdvBounds16 {
    static constexpr bool light = (FT & FT_LEAN) != 0 && (FT & FT_EXTRAS) == 0 &&
                                  (FT & (FT_COMP | FT_CURV)) != (FT_COMP | FT_CURV) &&
                                  (FT & (FT_CURV | FT_DEFER)) != 0;
    static constexpr int threads = light ? 128 : 256, blocks = light ? GR_F32_LIGHT_BLOCKS : GR_ADV_MIN_BLOCKS;
};
template <int FT> struct AdvBounds<3, Pair<__nv_bfloat16>, FT> : AdvBounds16<__nv_bfloat16, FT> {};
template <int FT> struct AdvBounds<3, Pair<__half>, FT> : AdvBounds16<__half, FT> {};
template <int FT> struct AdvBounds<3, Pair<float>, FT> {
    static constexpr bool light = (FT & FT_LEAN) != 0 && (FT & FT_EXTRAS) == 0 &&
                                  (FT & (FT_COMP | FT_CURV)) != (FT_COMP | FT_CURV);
    static constexpr int threads = 128, blocks = light ? GR_F32_LIGHT_BLOCKS : GR_F32_PAIR_BLOCKS;
};

template <int DIM, bool RK4, typename W, int FT>
__global__ void __launch_bounds__(AdvBounds<DIM, W, FT>::threads, AdvBounds<DIM, W, FT>::blocks)
    advance_kernel(const __grid_constant__ KParams P) {
    const int64_t n_live = P.n_dev ? (int64_t)*P.n_dev : P.n;
    unsigned long long steps = 0;
    unsigned alive = 0;
    if (P.grid_stride) {
        const int64_t stride = (int64_t)gridDim.x * blockDim.x;
        for (int64_t base = (int64_t)blockIdx.x * blockDim.x; base < n_live; base += stride)
            advance_particle<DIM, RK4, W, FT>(P, base + threadIdx.x, n_live, steps, alive);
    } else {
        advance_particle<DIM, RK4, W, FT>(P, (int64_t)blockIdx.x * blockDim.x + threadIdx.x, n_live, steps, alive);
    }
    // counters: particle-steps and the alive count after the launch (warp-aggregated)
    const unsigned long long warp_steps = __reduce_add_sync(0xffffffffu, (unsigned)steps);
    const unsigned warp_alive = __reduce_add_sync(0xffffffffu, alive);
    if ((threadIdx.x & 31) == 0) {
        if (warp_steps) atomicAdd(P.counters, warp_steps);
        if (warp_alive) atomicAdd(P.counters + 1, (unsigned long long)warp_alive);
    }
}

}  // namespace granite_b200
