// fvm2d_split.cuh -- the storage of the FP32 build with residual planes: a
// value x is kept as hi = x rounded to FP32 plus lo = (x - hi) rounded to
// bfloat16 (FP32's exponent range, 8 significant bits), so the stored value
// carries about 32 significant bits in 6 bytes.  A state buffer holds the 4
// FP32 planes (`plane` elements apart) followed by the residual block: for
// each element offset o of a plane, the 4 fields' residuals as one 8-byte
// word (16-bit residual of field f at index 4 o + f), so a sweep moves a
// cell's residuals with one load and one store.
#pragma once

#include <cuda_runtime.h>
#include <string.h>

namespace fvm2d {

// bfloat16 bits of f, rounded to nearest with ties to even: the upper 16 bits
// of f after adding half of the dropped part's unit (plus one when the kept
// part is odd).  The residuals this stores are finite and small, so NaN and
// overflow need no care here.
__host__ __device__ inline unsigned short bf16_bits(float f)
{
    unsigned int u;
    memcpy(&u, &f, 4);
    u += 0x7fffu + ((u >> 16) & 1u);
    return (unsigned short)(u >> 16);
}

__host__ __device__ inline float bf16_value(unsigned short b)
{
    const unsigned int u = (unsigned int)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// hi + lo of x (hi rounded to nearest; lo the rounded remainder).  Where
// the remainder rounds to half a unit of hi's last place, hi + lo lies
// halfway between two FP32 values and rounding it to FP32 picks the even
// one: that one is stored as hi (with the remainder taken from it), so that
// splitting hi + lo again gives the same hi and lo -- a state read back and
// set again continues bit for bit.  The stored value hi + lo is the same
// either way.
__host__ __device__ inline void split_value(double x, float &hi, unsigned short &lo)
{
    hi = float(x);
    lo = bf16_bits(float(x - double(hi)));
    const float even = float(double(hi) + double(bf16_value(lo)));
    if (even != hi) {
        hi = even;
        lo = bf16_bits(float(x - double(hi)));
    }
}

__host__ __device__ inline double join_value(float hi, unsigned short lo) { return double(hi) + double(bf16_value(lo)); }

// Element k of 4 state planes (k = field * plane + offset in the plane), for
// the transfer kernels: plain planes of T, or FP32 planes with residuals.
template <typename T>
struct Planes {
    T *U;
    __host__ __device__ double get(long long k) const { return double(U[k]); }
    __host__ __device__ void put(long long k, double v) const { U[k] = T(v); }
};

struct SplitPlanes {
    float *hi;
    unsigned short *lo;  // the residual block
    long long plane;
    __host__ __device__ long long lo_index(long long k) const
    {
        const long long f = k / plane;
        return 4 * (k - f * plane) + f;
    }
    __host__ __device__ double get(long long k) const { return join_value(hi[k], lo[lo_index(k)]); }
    __host__ __device__ void put(long long k, double v) const { split_value(v, hi[k], lo[lo_index(k)]); }
};

// The residual block of a state buffer of FP32 planes `plane` elements apart.
__host__ __device__ inline unsigned short *residual_block(void *state, long long plane)
{
    return reinterpret_cast<unsigned short *>(static_cast<float *>(state) + 4 * plane);
}

inline SplitPlanes split_planes(void *state, long long plane)
{
    return SplitPlanes{static_cast<float *>(state), residual_block(state, plane), plane};
}

} // namespace fvm2d
