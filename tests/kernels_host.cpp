// kernels_host.cpp -- the device code of the step's kernels compiled for the
// host with g++ from 2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh, so that the CPU
// tests can compare it with the oracle without a GPU: the ghost-ring rules
// (ghost_cell), the step-size plan (plan_step), the wave speed, and the sweep
// work items themselves (x_item, y_item) with the kernels' item numbering.
// tests/test_kernels_host.py builds it and calls it through ctypes.
//
// An x-sweep work item is warp-cooperative: its lanes pass slopes and fluxes
// to their neighbours with warp shuffles.  Here a warp is 32 host threads
// running the same item sequence; a shuffle is a barrier-separated exchange
// through a per-lane slot.  The block-level reductions and atomics of the
// kernels themselves are declared so that the header compiles; nothing called
// here reaches them.
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace warp_emu {
constexpr int kLanes = 32;
thread_local int lane_id = 0;
struct Barrier {
    std::mutex m;
    std::condition_variable cv;
    int count = 0, gen = 0;
    void wait()
    {
        std::unique_lock<std::mutex> l(m);
        const int g = gen;
        if (++count == kLanes) {
            count = 0;
            ++gen;
            cv.notify_all();
        } else {
            cv.wait(l, [&] { return gen != g; });
        }
    }
};
static Barrier bar;
static unsigned char slot[kLanes][16];

// value of lane (lane_id + delta), or the caller's own where that lane is
// outside the warp, as the hardware shuffles do
template <typename T>
T exchange(T v, int delta)
{
    static_assert(sizeof(T) <= sizeof(slot[0]), "shuffle operand too wide");
    std::memcpy(slot[lane_id], &v, sizeof(T));
    bar.wait();
    T r = v;
    const int src = lane_id + delta;
    if (src >= 0 && src < kLanes) std::memcpy(&r, slot[src], sizeof(T));
    bar.wait();
    return r;
}
} // namespace warp_emu

static inline double rsqrt(double x) { return 1.0 / std::sqrt(x); }
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }
static uint3 threadIdx, blockIdx;
static dim3 blockDim, gridDim;
template <typename T>
static inline T __shfl_xor_sync(unsigned, T v, int) { return v; }
template <typename T>
static inline T __shfl_down_sync(unsigned, T v, int d) { return warp_emu::exchange(v, d); }
template <typename T>
static inline T __shfl_up_sync(unsigned, T v, int d) { return warp_emu::exchange(v, -d); }
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

// One sweep of a (ny, nx, 4) state through the kernels' work items: dir 0
// runs x_item over every (row, 30-cell segment) item with a 32-thread warp,
// dir 1 runs y_item over every (32-column, T-interface segment) item, lane by
// lane (y items exchange nothing).  final (x only): the final sweep, which
// averages with `comb` (branch A) in place, as the kernel does: `out` starts
// as `comb` and is both read and written.  policy 0 = RefOrder, 1 = Hoisted.
// Cells the items do not write are left NaN in `out` (or `comb`'s values).
int kh_sweep(int policy, int dir, int final, int T, const double *in, const double *comb, double *out, int nx,
             int ny, double h, double dt, double alpha, double gamma)
{
    if (nx < 6 || ny < 6 || (dir == 1 && T < 3) || (final && dir != 0)) return 1;
    const long long plane = (long long)nx * ny;
    if (final && !comb) return 1;
    std::vector<double> S(4 * plane), D(4 * plane, NAN);
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) {
            S[f * plane + c] = in[4 * c + f];
            if (final) D[f * plane + c] = comb[4 * c + f];
        }
    SweepArgs<double> a;
    a.src = Field<double>{S.data(), plane, nx};
    a.dst = Field<double>{D.data(), plane, nx};
    a.comb = a.dst;
    a.flux = Field<double>{nullptr, plane, nx};
    a.nx = nx;
    a.ny = ny;
    a.h = h;
    a.rh = 1.0 / h;
    a.alpha = alpha;
    a.gamma = gamma;
    a.ctl = nullptr;
    const SweepConsts<double> K = sweep_consts(a, dt);
    if (dir == 0) {
        const int nseg = (nx - 4 + kXCells - 1) / kXCells;
        const long long nwork = (long long)nseg * ny;
        auto lane_run = [&](int lane) {
            warp_emu::lane_id = lane;
            double vmax = 0.0;
            int bad = 0;
            for (long long w = 0; w < nwork; ++w) {
                const int y = int(w / nseg), seg = int(w % nseg);
                if (policy == 0 && final)
                    x_item<double, RefOrder, true>(a, K, y, seg, nseg, lane, vmax, bad);
                else if (policy == 0)
                    x_item<double, RefOrder, false>(a, K, y, seg, nseg, lane, vmax, bad);
                else if (final)
                    x_item<double, Hoisted, true>(a, K, y, seg, nseg, lane, vmax, bad);
                else
                    x_item<double, Hoisted, false>(a, K, y, seg, nseg, lane, vmax, bad);
            }
        };
        std::vector<std::thread> warp;
        for (int lane = 0; lane < warp_emu::kLanes; ++lane) warp.emplace_back(lane_run, lane);
        for (auto &th : warp) th.join();
    } else {
        const int ncw = (nx + 31) / 32, nseg = y_segments(ny, T);
        for (int seg = 0; seg < nseg; ++seg)
            for (int cw = 0; cw < ncw; ++cw)
                for (int lane = 0; lane < 32; ++lane) {
                    if (policy == 0)
                        y_item<double, RefOrder>(a, K, seg, nseg, cw, lane, T);
                    else
                        y_item<double, Hoisted>(a, K, seg, nseg, cw, lane, T);
                }
    }
    for (long long c = 0; c < plane; ++c)
        for (int f = 0; f < 4; ++f) out[4 * c + f] = D[f * plane + c];
    return 0;
}

} // extern "C"
