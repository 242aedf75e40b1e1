// kernels_host.cpp -- the parts of the sweep kernels' device code that run
// one thread per cell with no exchange between threads -- the ghost-ring
// rules (ghost_cell), the step-size plan (plan_step) and the wave speed --
// compiled for the host with g++ from 2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh,
// so that the CPU tests can compare them with the oracle on every preset and
// slab row frame.  tests/test_kernels_host.py builds it and calls it through
// ctypes.
//
// The rest of fvm2d_kernels.cuh uses warp, block and atomic intrinsics that
// exist only in device code; they are declared below so that the header
// compiles, and nothing called here reaches them.
#include <cmath>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
static uint3 threadIdx, blockIdx;
static dim3 blockDim, gridDim;
template <typename T>
static inline T __shfl_xor_sync(unsigned, T v, int) { return v; }
template <typename T>
static inline T __shfl_down_sync(unsigned, T v, int) { return v; }
template <typename T>
static inline T __shfl_up_sync(unsigned, T v, int) { return v; }
template <typename T>
static inline T __shfl_sync(unsigned, T v, int) { return v; }
static inline void __syncthreads() {}
static inline void __threadfence() {}
static inline int __any_sync(unsigned, int p) { return p; }
static inline long long __double_as_longlong(double x)
{
    long long r;
    std::memcpy(&r, &x, 8);
    return r;
}
static inline double __longlong_as_double(long long x)
{
    double r;
    std::memcpy(&r, &x, 8);
    return r;
}
template <typename T>
static inline T atomicAdd(T *p, T v)
{
    const T o = *p;
    *p = o + v;
    return o;
}
template <typename T>
static inline T atomicMax(T *p, T v)
{
    const T o = *p;
    if (v > o) *p = v;
    return o;
}
template <typename T>
static inline T atomicCAS(T *p, T c, T v)
{
    const T o = *p;
    if (o == c) *p = v;
    return o;
}
#pragma GCC diagnostic ignored "-Wunknown-pragmas"
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }
#define __launch_bounds__(...)

#define FVM2D_VARIANT host
#include "../2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh"

using namespace fvm2d::host;
using fvm2d::PlanParams;
using fvm2d::StepControl;

extern "C" {

// The ghost fill of ghost_kernel on a (ny, nx, 4) array of (rho, p, u, v)
// cells, in place: every ring cell from ghost_cell at time t in the row frame
// (row0, gny, fill_top, fill_bottom).  *vmax: the ring cells' largest wave
// speed, as the kernel folds it into the step's maximum.
int kh_ghost(double *cells, int nx, int ny, int strategy, double gamma, double t, int row0, int gny, int fill_top,
             int fill_bottom, double *vmax)
{
    if (nx < 6 || ny < 6) return 1;
    const long long plane = (long long)nx * ny;
    std::vector<double> P(4 * plane);
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) P[f * plane + c] = cells[4 * c + f];
    GhostArgs<double> a;
    a.U.base = P.data();
    a.U.plane = plane;
    a.U.pitch = nx;
    a.nx = nx;
    a.ny = ny;
    a.strategy = strategy;
    a.gamma = gamma;
    a.ctl = nullptr;
    a.plan = PlanParams{};
    a.row0 = row0;
    a.gny = gny;
    a.fill_top = fill_top;
    a.fill_bottom = fill_bottom;
    double m = 0.0;
    for (int k = 0; k < 4 * nx + 4 * (ny - 4); ++k) m = std::fmax(m, ghost_cell(a, k, t));
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) cells[4 * c + f] = P[f * plane + c];
    *vmax = m;
    return 0;
}

// plan_step on a control record with committed time t, wave-speed max smax,
// `steps` of `step_limit` and the done flag.  out: dt, active, done.
int kh_plan(double t, double smax, int steps, int step_limit, int done, double t_end, double cfl, double hmin,
            double fixed_dt, double *dt, int *active, int *done_out)
{
    StepControl c{};
    c.t = t;
    c.smax_last = smax;
    c.steps = steps;
    c.step_limit = step_limit;
    c.done = done;
    c.dt = -1.0;
    PlanParams p{t_end, cfl, hmin, fixed_dt};
    plan_step(&c, p);
    *dt = c.dt;
    *active = c.active;
    *done_out = c.done;
    return 0;
}

// Wave speed |(u, v)| + sqrt(gamma p / rho) of n cells (n x 4).
int kh_wave_speed(long n, const double *cells, double gamma, double *out)
{
    for (long i = 0; i < n; ++i) {
        const double *c = cells + 4 * i;
        out[i] = wave_speed(c[0], c[1], c[2], c[3], gamma);
    }
    return 0;
}

} // extern "C"
