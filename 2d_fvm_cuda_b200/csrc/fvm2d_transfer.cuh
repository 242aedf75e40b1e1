// fvm2d_transfer.cuh -- state transfers shared by the solver and batch host
// runtimes: host cells (stride doubles each, row-major) <-> device planes.
// The planes are reached through a storage policy S (fvm2d_split.cuh):
// Planes<double>, Planes<float>, or SplitPlanes (FP32 with residual planes),
// whose get/put convert element k to and from double.
#pragma once

#include <cuda_runtime.h>

#include "fvm2d_split.cuh"

namespace fvm2d {

// AoS (stride doubles per cell, row-major) <-> SoA planes with a row pitch.
template <class S>
static __global__ void aos_to_soa(const double *__restrict__ in, int stride, S U, int nx, int ny, int pitch,
                                  long long plane)
{
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = int(k / nx), x = int(k % nx);
        const long long o = (long long)y * pitch + x;
        for (int f = 0; f < 4; ++f) U.put(f * plane + o, in[k * stride + f]);
    }
}

template <class S>
static __global__ void soa_to_aos(S U, int nx, int ny, int pitch, long long plane, int stride, double *__restrict__ out)
{
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = int(k / nx), x = int(k % nx);
        const long long o = (long long)y * pitch + x;
        for (int f = 0; f < 4; ++f) out[k * stride + f] = U.get(f * plane + o);
        for (int f = 4; f < stride; ++f) out[k * stride + f] = 0.0;
    }
}

// Element-wise conversion of the 4 state planes (n = 4 plane elements)
// between storage policies.
template <class S, class D>
static __global__ void convert_planes(S in, D out, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        out.put(k, in.get(k));
}

// Rows j0 .. j0+nrows-1 of the four planes, packed as [4][nrows][nx] doubles
// (rows_out) and back (rows_in).
template <class S>
static __global__ void rows_out(S U, long long plane, int pitch, int j0, int nrows, int nx, double *__restrict__ out)
{
    const long long per = (long long)nrows * nx, n = 4 * per;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int f = int(k / per), r = int(k % per / nx), x = int(k % nx);
        out[k] = U.get(f * plane + (long long)(j0 + r) * pitch + x);
    }
}

template <class S>
static __global__ void rows_in(S U, long long plane, int pitch, int j0, int nrows, int nx, const double *__restrict__ in)
{
    const long long per = (long long)nrows * nx, n = 4 * per;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int f = int(k / per), r = int(k % per / nx), x = int(k % nx);
        U.put(f * plane + (long long)(j0 + r) * pitch + x, in[k]);
    }
}

inline bool is_device_pointer(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

} // namespace fvm2d
