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

// Conserved totals of the interior cells (rows and columns 2 .. n-3, the
// cells the sweeps update): per block, the sums of rho, rho u, rho v and
// E = p / (gamma - 1) + rho (u^2 + v^2) / 2 in FP64 whatever the storage,
// written to partial[4 * block + f]; conserved_sum then adds the blocks in
// block order.  Cells are dealt to threads by a fixed grid-stride and the
// block sums follow a fixed tree, so a state gives the same bits on every
// call with the same grid.  NT is the block size (a power of two).
template <class S, int NT>
static __global__ void __launch_bounds__(NT) conserved_partials(S U, int nx, int ny, int pitch, long long plane,
                                                                double gamma, double *__restrict__ partial)
{
    __shared__ double red[4][NT];
    const int t = threadIdx.x;
    const int iw = nx - 4;
    const long long n = (long long)iw * (ny - 4);
    const double igm1 = 1.0 / (gamma - 1.0);
    double m = 0.0, mu = 0.0, mv = 0.0, e = 0.0;
    for (long long k = blockIdx.x * (long long)NT + t; k < n; k += (long long)gridDim.x * NT) {
        const long long o = (long long)(2 + k / iw) * pitch + (2 + k % iw);
        const double rho = U.get(o), p = U.get(plane + o), u = U.get(2 * plane + o), v = U.get(3 * plane + o);
        m += rho;
        mu += rho * u;
        mv += rho * v;
        e += p * igm1 + 0.5 * rho * (u * u + v * v);
    }
    red[0][t] = m;
    red[1][t] = mu;
    red[2][t] = mv;
    red[3][t] = e;
    __syncthreads();
    for (int s = NT / 2; s > 0; s >>= 1) {
        if (t < s)
            for (int f = 0; f < 4; ++f) red[f][t] += red[f][t + s];
        __syncthreads();
    }
    if (t < 4) partial[4 * blockIdx.x + t] = red[t][0];
}

// totals[f] = area * sum over blocks b (in order) of partial[4 b + f]; one
// thread per total.
static __global__ void conserved_sum(const double *__restrict__ partial, int nblocks, double area,
                                     double *__restrict__ totals)
{
    const int f = threadIdx.x;
    if (f >= 4) return;
    double s = 0.0;
    for (int b = 0; b < nblocks; ++b) s += partial[4 * b + f];
    totals[f] = s * area;
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
