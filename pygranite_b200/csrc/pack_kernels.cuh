// pack_kernels.cuh — snapshot packing shared by the engine (engine.cu) and the request
// server (server.cu): float32 planes -> the node-major storage layout of the device ring, and
// two ring slots -> the window-pair buffer the step kernel reads.  Internal linkage: each
// translation unit that includes this header owns its instances (static kernels).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <cstdint>

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

// 2D window pair with replicated edges: padded node (x, y), x in [-1, nx + 1], y in [-1, ny + 1],
// of a (nx + 3) x (ny + 3) buffer holds the back slot's node (clamp(x), clamp(y)) followed by the
// front slot's (the step kernel's clamp addressing).  T is one packed node (8 bytes float32, 4
// bytes 16-bit); every padded node is written.
template <typename T>
static __global__ void pair_pack_edge2_kernel(const T *__restrict__ back, const T *__restrict__ front, T *out,
                                              int32_t nx, int32_t ny) {
    const int32_t pnx = nx + 3;
    const int32_t total = pnx * (ny + 3);
    for (int32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
        const int32_t x = min(max(o % pnx - 1, 0), nx - 1), y = min(max(o / pnx - 1, 0), ny - 1);
        const int64_t i = (int64_t)y * nx + x;
        out[2 * (int64_t)o] = back[i];
        out[2 * (int64_t)o + 1] = front[i];
    }
}

// 3D window pair with a zero border: padded node (x, y, z), x in [-1, nx + 1] and likewise y,
// z, of a (nx + 3) x (ny + 3) x (nz + 3) buffer holds the back slot's node (x, y, z) followed by
// the front slot's, or zeros outside the grid (the step kernel's border addressing).  T is one
// packed node (16 bytes float32, 8 bytes 16-bit); every padded node is written, so the buffer
// needs no clearing.  The padded node count must stay below 2^31.
template <typename T>
static __global__ void pair_pack_padded_kernel(const T *__restrict__ back, const T *__restrict__ front, T *out,
                                               int32_t nx, int32_t ny, int32_t nz) {
    const int32_t pnx = nx + 3, pny = ny + 3;
    const int32_t total = pnx * pny * (nz + 3);
    for (int32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < total; o += gridDim.x * blockDim.x) {
        const int32_t x = o % pnx - 1, r = o / pnx;
        const int32_t y = r % pny - 1, z = r / pny - 1;
        T b{}, f{};
        if ((unsigned)x < (unsigned)nx && (unsigned)y < (unsigned)ny && (unsigned)z < (unsigned)nz) {
            const int64_t i = ((int64_t)z * ny + y) * nx + x;
            b = back[i];
            f = front[i];
        }
        out[2 * (int64_t)o] = b;
        out[2 * (int64_t)o + 1] = f;
    }
}

}  // namespace granite_b200
