// fvm2d_split.cuh -- the storage of the FP32 build with residual planes: a
// value x is kept as hi = x rounded to FP32 plus lo = (x - hi) cut to
// bfloat16 (FP32's exponent range, 8 significant bits), so the stored value
// carries about 31 significant bits in 6 bytes.  A state buffer holds the 4
// FP32 planes (`plane` elements apart) followed by the residual block: for
// each element offset o of a plane, the 4 fields' residuals as one 8-byte
// word (16-bit residual of field f at index 4 o + f), so a sweep moves a
// cell's residuals with one load and one store.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

namespace fvm2d {

// bfloat16 value of 16 bits: the upper half of an FP32 value.
__host__ __device__ inline float bf16_value(unsigned short b)
{
    const unsigned int u = (unsigned int)b << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// hi + lo of x: hi = x rounded to nearest FP32; lo = x - hi (exact in FP64)
// rounded toward zero to FP32 and truncated to bfloat16 (its upper 16 bits).
// |lo| then stays below half a unit of hi's last place (or equals it where
// x itself lies halfway, hi then even), so hi + lo rounds back to hi and
// splitting it again gives the same hi and lo: a state read back and set
// again continues bit for bit.  |x - (hi + lo)| < 2^-31 |x|.
__host__ __device__ inline void split_value(double x, float &hi, unsigned short &lo)
{
    hi = float(x);
    const double r = x - double(hi);
#if defined(__CUDA_ARCH__)
    const float rf = __double2float_rz(r);
#else
    float rf = float(r);
    if (fabs(double(rf)) > fabs(r)) rf = nextafterf(rf, 0.0f);
#endif
    unsigned int u;
    memcpy(&u, &rf, 4);
    lo = (unsigned short)(u >> 16);
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
