// pack_kernels.cuh — snapshot packing shared by the engine (engine.cu) and the request
// server (server.cu): float32 planes -> the node-major storage layout of the device ring, and
// two ring slots -> the window-pair buffer the step kernel reads.  Internal linkage: each
// translation unit that includes this header owns its instances (static kernels).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

namespace granite_b200 {

// Planes (ncomp x nodes, float32) -> node-major packed snapshot of storage type W.
template <typename W>
static __global__ void pack_wind_kernel(const float *__restrict__ u, const float *__restrict__ v,
                                 const float *__restrict__ w, void *out, int64_t nodes, int dim);

template <>
__global__ void pack_wind_kernel<float>(const float *__restrict__ u, const float *__restrict__ v,
                                        const float *__restrict__ w, void *out, int64_t nodes, int dim) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        if (dim == 3) reinterpret_cast<float4 *>(out)[i] = make_float4(u[i], v[i], w[i], 0.f);
        else reinterpret_cast<float2 *>(out)[i] = make_float2(u[i], v[i]);
    }
}

template <>
__global__ void pack_wind_kernel<__nv_bfloat16>(const float *__restrict__ u, const float *__restrict__ v,
                                                const float *__restrict__ w, void *out, int64_t nodes, int dim) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const __nv_bfloat162 a = __floats2bfloat162_rn(u[i], v[i]);
        if (dim == 3) {
            const __nv_bfloat162 b = __floats2bfloat162_rn(w[i], 0.f);
            uint2 q;
            q.x = *reinterpret_cast<const unsigned *>(&a);
            q.y = *reinterpret_cast<const unsigned *>(&b);
            reinterpret_cast<uint2 *>(out)[i] = q;
        } else {
            reinterpret_cast<unsigned *>(out)[i] = *reinterpret_cast<const unsigned *>(&a);
        }
    }
}

template <>
__global__ void pack_wind_kernel<__half>(const float *__restrict__ u, const float *__restrict__ v,
                                         const float *__restrict__ w, void *out, int64_t nodes, int dim) {
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nodes; i += (int64_t)gridDim.x * blockDim.x) {
        const __half2 a = __floats2half2_rn(u[i], v[i]);
        if (dim == 3) {
            const __half2 b = __floats2half2_rn(w[i], 0.f);
            uint2 q;
            q.x = *reinterpret_cast<const unsigned *>(&a);
            q.y = *reinterpret_cast<const unsigned *>(&b);
            reinterpret_cast<uint2 *>(out)[i] = q;
        } else {
            reinterpret_cast<unsigned *>(out)[i] = *reinterpret_cast<const unsigned *>(&a);
        }
    }
}

// The window pair interleaves the two snapshots component by component (granite_kernels.cuh,
// Store<Pair<...>>): from ring nodes b (back) and f (front) of storage type S to one pair node.
// float32: ring nodes float4 {u, v, w, 0} / float2 {u, v}; 16-bit: uint2 {(u, v), (w, 0)} /
// one word (u, v), each word two 16-bit values (low half first).
template <typename S> struct PairNode;

template <> struct PairNode<float> {
    using Ring3 = float4;
    using Ring2 = float2;
    using Out3 = uint4;   // written as two of these: 32 bytes
    using Out2 = float4;
    static __device__ __forceinline__ void pack3(const float4 &b, const float4 &f, float4 *o) {
        o[0] = make_float4(b.x, f.x, b.y, f.y);
        o[1] = make_float4(b.z, f.z, 0.f, 0.f);
    }
    static __device__ __forceinline__ float4 pack2(const float2 &b, const float2 &f) { return make_float4(b.x, f.x, b.y, f.y); }
};

template <> struct PairNode<uint16_t> {
    using Ring3 = uint2;
    using Ring2 = unsigned;
    using Out2 = uint2;
    // __byte_perm(x, y, 0x5410): the low halves of x and y; 0x7632: their high halves
    static __device__ __forceinline__ uint4 pack3(const uint2 &b, const uint2 &f) {
        return make_uint4(__byte_perm(b.x, f.x, 0x5410), __byte_perm(b.x, f.x, 0x7632), __byte_perm(b.y, f.y, 0x5410), 0u);
    }
    static __device__ __forceinline__ uint2 pack2(unsigned b, unsigned f) {
        return make_uint2(__byte_perm(b, f, 0x5410), __byte_perm(b, f, 0x7632));
    }
};

// 2D window pair with replicated edges: padded node (x, y), x in [-1, nx + 1], y in [-1, ny + 1],
// of a (nx + 3) x (ny + 3) buffer holds the pair of ring nodes (clamp(x), clamp(y)) (the step
// kernel's clamp addressing).  Every padded node is written.
template <typename S>
static __global__ void pair_pack_edge2_kernel(const typename PairNode<S>::Ring2 *__restrict__ back,
                                              const typename PairNode<S>::Ring2 *__restrict__ front,
                                              typename PairNode<S>::Out2 *out, int32_t nx, int32_t ny) {
    const int32_t pnx = nx + 3;
    const int32_t total = pnx * (ny + 3);
    for (int32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
        const int32_t x = min(max(o % pnx - 1, 0), nx - 1), y = min(max(o / pnx - 1, 0), ny - 1);
        const int64_t i = (int64_t)y * nx + x;
        out[o] = PairNode<S>::pack2(back[i], front[i]);
    }
}

// 3D window pair with a zero border: padded node (x, y, z), x in [-1, nx + 1] and likewise y, z,
// of a (nx + 3) x (ny + 3) x (nz + 3) buffer holds the pair of ring nodes (x, y, z), or zeros
// outside the grid (the step kernel's border addressing).  Every padded node is written, so the
// buffer needs no clearing.  The padded node count must stay below 2^31.
// 128-thread blocks, 4 nodes in flight per thread.  (Run as one 32-register block per SM beside
// the step launches, the pack measured 1% faster on the 3D benchmark configuration and 3-15%
// slower on the other 3D configurations, so it covers the whole buffer at once.)
constexpr int PACK3_THREADS = 128, PACK3_UNROLL = 4;
template <typename S>
static __global__ void __launch_bounds__(PACK3_THREADS, 16)
    pair_pack_padded_kernel(const typename PairNode<S>::Ring3 *__restrict__ back,
                            const typename PairNode<S>::Ring3 *__restrict__ front, void *__restrict__ out, int32_t nx,
                            int32_t ny, int32_t nz) {
    const int32_t pnx = nx + 3, pny = ny + 3;
    const int32_t total = pnx * pny * (nz + 3);
    const int32_t chunk = PACK3_THREADS * PACK3_UNROLL;
    for (int32_t o0 = blockIdx.x * chunk + threadIdx.x; o0 < total; o0 += gridDim.x * chunk) {
#pragma unroll
        for (int u = 0; u < PACK3_UNROLL; ++u) {
            const int32_t o = o0 + u * PACK3_THREADS;
            if (o >= total) break;
            const int32_t x = o % pnx - 1, r = o / pnx;
            const int32_t y = r % pny - 1, z = r / pny - 1;
            const bool in = (unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz;
            const int64_t i = in ? ((int64_t)z * ny + y) * nx + x : 0;
            if constexpr (std::is_same<S, float>::value) {
                float4 *po = reinterpret_cast<float4 *>(out) + 2 * (int64_t)o;
                if (in) {
                    PairNode<float>::pack3(back[i], front[i], po);
                } else {
                    po[0] = make_float4(0.f, 0.f, 0.f, 0.f);
                    po[1] = make_float4(0.f, 0.f, 0.f, 0.f);
                }
            } else {
                reinterpret_cast<uint4 *>(out)[o] = in ? PairNode<uint16_t>::pack3(back[i], front[i]) : make_uint4(0u, 0u, 0u, 0u);
            }
        }
    }
}

}  // namespace granite_b200
