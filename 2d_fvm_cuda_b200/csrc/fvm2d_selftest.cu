// fvm2d_selftest.cu -- evaluates the refined reciprocal and reciprocal
// square root of the FP64 product build (rrcp / rrsqrt of fvm2d_math.cuh,
// compiled here exactly as in that build) on caller-given arguments, so
// tests can hold them to their error bound against correctly rounded values.
#define FVM2D_VARIANT selftest
#define FVM2D_FAST_RCP
#include "../../include/fvm2d.h"
#include "fvm2d_control.h"
#include "fvm2d_math.cuh"

#include <string>

namespace {

__global__ void eval_reciprocals(const double *__restrict__ x, long long n, double *__restrict__ rcp,
                                 double *__restrict__ rsq)
{
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        rcp[k] = fvm2d::selftest::rrcp(x[k]);
        rsq[k] = fvm2d::selftest::rrsqrt(x[k]);
    }
}

} // namespace

extern "C" {
#pragma GCC visibility push(default)

int fvm2d_eval_reciprocals(const double *x, long long n, double *rcp, double *rsqrt_out)
{
    if (n < 0 || (n > 0 && (!x || !rcp || !rsqrt_out)))
        return fvm2d::report_error(FVM2D_ERR_INVALID, "null pointer or negative count");
    if (n == 0) return FVM2D_OK;
    const int threads = 256;
    const long long want = (n + threads - 1) / threads;
    eval_reciprocals<<<(int)(want < 4096 ? want : 4096), threads>>>(x, n, rcp, rsqrt_out);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fvm2d::report_error(FVM2D_ERR_CUDA, (std::string("reciprocal kernel: ") + cudaGetErrorString(e)).c_str());
    }
    return FVM2D_OK;
}

#pragma GCC visibility pop
} // extern "C"
