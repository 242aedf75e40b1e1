// fvm2d_dual.cuh -- first-order dual numbers (value + tangent) for the
// tangent-linear (JVP) build of the kernels.
//
// The type and its functions live in namespace fvm2d::ad and are found by
// argument-dependent lookup, so unqualified sqrt/fabs on plain doubles keep
// resolving to the standard functions.
//
// Instantiating the templated sweep, ghost and update code with Real = Dual
// propagates a tangent alongside every value through exactly the arithmetic
// the FP64 build performs.  Comparisons and branches act on values, so the
// derivative taken is that of the branch the value selects (the almost-
// everywhere derivative through the limiter's min/max and sign tests and the
// Riemann solver's wave cases).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace fvm2d {
namespace ad {

struct Dual {
    double v, d;
    __host__ __device__ Dual() : v(0.0), d(0.0) {}
    __host__ __device__ Dual(double value) : v(value), d(0.0) {}
    __host__ __device__ Dual(double value, double tangent) : v(value), d(tangent) {}
    __host__ __device__ explicit operator double() const { return v; }
};

__host__ __device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__host__ __device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__host__ __device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__host__ __device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__host__ __device__ __forceinline__ Dual operator/(Dual a, Dual b)
{
    const double q = a.v / b.v;
    return Dual(q, (a.d - q * b.d) / b.v);
}
__host__ __device__ __forceinline__ Dual &operator+=(Dual &a, Dual b) { return a = a + b; }
__host__ __device__ __forceinline__ Dual &operator-=(Dual &a, Dual b) { return a = a - b; }
__host__ __device__ __forceinline__ Dual &operator*=(Dual &a, Dual b) { return a = a * b; }
__host__ __device__ __forceinline__ bool operator<(Dual a, Dual b) { return a.v < b.v; }
__host__ __device__ __forceinline__ bool operator>(Dual a, Dual b) { return a.v > b.v; }
__host__ __device__ __forceinline__ bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
__host__ __device__ __forceinline__ bool operator>=(Dual a, Dual b) { return a.v >= b.v; }

__device__ __forceinline__ Dual sqrt(Dual a)
{
    const double r = ::sqrt(a.v);
    return Dual(r, a.d / (2.0 * r));
}
__device__ __forceinline__ Dual rrsqrt(Dual a)
{
    const double r = ::rsqrt(a.v);
    return Dual(r, -0.5 * r * r * r * a.d);
}
__device__ __forceinline__ Dual fabs(Dual a) { return a.v < 0.0 ? -a : a; }
__device__ __forceinline__ Dual fma(Dual a, Dual b, Dual c) { return a * b + c; }

// Warp shuffles of a dual move both parts.
__device__ __forceinline__ Dual lane_down(Dual a)
{
    return Dual(__shfl_down_sync(0xffffffffu, a.v, 1), __shfl_down_sync(0xffffffffu, a.d, 1));
}
__device__ __forceinline__ Dual lane_last(Dual a)
{
    return Dual(__shfl_sync(0xffffffffu, a.v, 31), __shfl_sync(0xffffffffu, a.d, 31));
}
__device__ __forceinline__ Dual lane_up(Dual a)
{
    return Dual(__shfl_up_sync(0xffffffffu, a.v, 1), __shfl_up_sync(0xffffffffu, a.d, 1));
}

} // namespace ad
} // namespace fvm2d
