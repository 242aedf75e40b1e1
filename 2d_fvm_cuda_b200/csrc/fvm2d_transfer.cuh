// fvm2d_transfer.cuh -- state transfers shared by the solver and batch host
// runtimes: host cells (stride doubles each, row-major) <-> device planes.
#pragma once

#include <cuda_runtime.h>

namespace fvm2d {

// AoS (stride doubles per cell, row-major) <-> SoA planes of T with a row pitch.
template <typename T>
static __global__ void aos_to_soa(const double *__restrict__ in, int stride, T *__restrict__ U, int nx, int ny, int pitch,
                           long long plane)
{
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = int(k / nx), x = int(k % nx);
        const long long o = (long long)y * pitch + x;
        for (int f = 0; f < 4; ++f) U[f * plane + o] = T(in[k * stride + f]);
    }
}

template <typename T>
static __global__ void soa_to_aos(const T *__restrict__ U, int nx, int ny, int pitch, long long plane, int stride,
                           double *__restrict__ out)
{
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int y = int(k / nx), x = int(k % nx);
        const long long o = (long long)y * pitch + x;
        for (int f = 0; f < 4; ++f) out[k * stride + f] = double(U[f * plane + o]);
        for (int f = 4; f < stride; ++f) out[k * stride + f] = 0.0;
    }
}

// Element-wise conversion of the 4 state planes between storage types.
template <typename S, typename D>
static __global__ void convert_planes(const S *__restrict__ in, D *__restrict__ out, long long n)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        out[k] = D(in[k]);
}

// Rows j0 .. j0+nrows-1 of the four planes, packed as [4][nrows][nx] doubles
// (rows_out) and back (rows_in).
template <typename T>
static __global__ void rows_out(const T *__restrict__ U, long long plane, int pitch, int j0, int nrows, int nx,
                                double *__restrict__ out)
{
    const long long per = (long long)nrows * nx, n = 4 * per;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int f = int(k / per), r = int(k % per / nx), x = int(k % nx);
        out[k] = double(U[f * plane + (long long)(j0 + r) * pitch + x]);
    }
}

template <typename T>
static __global__ void rows_in(T *__restrict__ U, long long plane, int pitch, int j0, int nrows, int nx,
                               const double *__restrict__ in)
{
    const long long per = (long long)nrows * nx, n = 4 * per;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const int f = int(k / per), r = int(k % per / nx), x = int(k % nx);
        U[f * plane + (long long)(j0 + r) * pitch + x] = T(in[k]);
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
