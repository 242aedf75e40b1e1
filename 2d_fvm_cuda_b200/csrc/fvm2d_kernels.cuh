// fvm2d_kernels.cuh -- the sm_100a kernels of one split step.
//
// A step is  U <- ghost( (Y(X(U)) + X(Y(U))) / 2 )  with one dt
// (src/wrappers.cuh:196-284).  It runs as five kernels, all reading the step
// size from a device-resident control record so the loop never waits on the
// host:
//
//   sweep<X>        U -> A         first sweep of branch A
//   sweep<Y>        U -> B         first sweep of branch B
//   sweep<Y>        A -> U         second sweep of branch A (U^n is dead now)
//   sweep<X,final>  B -> U         second sweep of branch B, fused with the
//                                  primitive average against U (branch A) and
//                                  the wave-speed max of the interior cells
//   ghost_fill      U -> U         boundary ring for the preset, wave-speed
//                                  max of the ring, and (last block) the time
//                                  advance plus the next step's dt
//
// Each sweep stages a tile of cells with a two-cell halo along the sweep
// line in shared memory, computes every limited slope once, every interface
// (relaxation GRP + midpoint flux) once, and every cell update once; the
// reference's slope, face-state, interface and transposed buffers never
// reach HBM.  The y-sweep indexes rows in reverse (line position l = ny-1-j)
// with (un, ut) = (v, u), which is the reference's anti-transpose
// (src/basicFuns.cuh:249-262) applied inside the tile instead of through
// global memory.
#pragma once

#include "fvm2d_control.h"
#include "fvm2d_math.cuh"

#include <stdint.h>

namespace fvm2d {
namespace FVM2D_VARIANT {

// Start the next step if the loop of wrappers.cuh:196-207 continues:
// dt = min(CFL h / smax, t_end - t); stop when t >= t_end or h/smax < 1e-20.
__device__ __forceinline__ void plan_step(StepControl *c, const PlanParams &p)
{
    c->active = 0;
    if (c->done) return;
    if (c->steps >= c->step_limit) return;
    const double t = c->t;
    if (!(t < p.t_end)) {
        c->done = 1;
        return;
    }
    const double smax = c->smax_last;
    const double a = p.cfl * p.hmin / smax, b = p.t_end - t;
    const double dt = (b < a) ? b : a;
    if (p.hmin / smax < 1e-20) {
        c->done = 1;
        return;
    }
    c->dt = dt;
    c->active = 1;
}

__global__ void plan_kernel(StepControl *c, PlanParams p)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) plan_step(c, p);
}

// Block-wide max of a non-negative double, folded into *bits with one atomic
// per block.  Values that are NaN never win (the running max ignores them).
template <int NT>
__device__ __forceinline__ void block_max_to(double v, unsigned long long *bits)
{
    __shared__ double red[NT / 32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < NT / 32) ? red[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
        if (lane == 0 && v > 0.0) atomicMax(bits, (unsigned long long)__double_as_longlong(v));
    }
}

// True in exactly one thread of the last block of the grid to get here, after
// every earlier block's global writes are visible.
__device__ __forceinline__ bool last_block_done(unsigned int *ticket)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned int k = atomicAdd(ticket, 1u);
        last = (k == gridDim.x * gridDim.y - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        return true;
    }
    return false;
}

template <typename Real>
struct Field {
    Real *base;     // plane 0; planes rho, p, u, v follow at `plane` elements
    long long plane;
    int pitch;
    __device__ __forceinline__ Real &at(int f, int x, int y) const
    {
        return base[(long long)f * plane + (long long)y * pitch + x];
    }
};

template <typename Real>
struct SweepArgs {
    Field<Real> src;   // state swept
    Field<Real> dst;   // result
    Field<Real> comb;  // final sweep only: branch-A result averaged in (may alias dst)
    int nx, ny;
    double h;          // spacing along the sweep
    double rh;         // 1.0 / h, as the reference computes it
    double alpha, gamma;
    StepControl *ctl;
};

// Wave speed of all cells of the initial state, then the first step's plan.
template <typename Real, int NT>
__global__ void __launch_bounds__(NT) init_kernel(Field<Real> U, int nx, int ny, double gamma,
                                                  StepControl *ctl, PlanParams p)
{
    double m = 0.0;
    const long long n = (long long)nx * ny;
    for (long long k = blockIdx.x * (long long)NT + threadIdx.x; k < n; k += (long long)gridDim.x * NT) {
        int y = int(k / nx), x = int(k % nx);
        m = fmax(m, wave_speed(U.at(0, x, y), U.at(1, x, y), U.at(2, x, y), U.at(3, x, y), gamma));
    }
    block_max_to<NT>(m, &ctl->smax_bits);
    if (last_block_done(&ctl->ticket)) {
        volatile StepControl *vc = ctl;
        ctl->smax_last = __longlong_as_double((long long)vc->smax_bits);
        ctl->smax_bits = 0ull;
        ctl->ticket = 0u;
        plan_step(ctl, p);
    }
}

// ---------------------------------------------------------------------------
// Sweep kernel.
//
// DIR 0: x-sweep; a tile is NL rows x TL interfaces along x.
// DIR 1: y-sweep; a tile is NL columns x TL interfaces along y.
// Tile t covers updated line positions [2 + t(TL-1), 2 + t(TL-1) + TL-1)
// and reads positions [l0-2, l0+TL].  Shared memory is laid out so that the
// x index is the fastest-varying one in both directions, keeping global
// loads and stores coalesced.
// ---------------------------------------------------------------------------
template <int DIR, int TL, int NL>
struct TileMap {
    // (line offset p in [0, len), cross c in [0, NL)) <-> flat index
    __device__ static __forceinline__ int idx(int p, int c, int len)
    {
        return DIR == 0 ? c * len + p : p * NL + c;
    }
    __device__ static __forceinline__ void split(int w, int len, int &p, int &c)
    {
        if (DIR == 0) { p = w % len; c = w / len; }
        else { c = w % NL; p = w / NL; }
    }
};

template <typename Real, int TL, int NL>
struct SweepSmem {
    static constexpr int CELLS = (TL + 3) * NL;
    static constexpr int SLOPES = (TL + 1) * NL;
    static constexpr int FLUXES = TL * NL;
    static constexpr size_t BYTES = sizeof(Real) * 4 * (CELLS + SLOPES + FLUXES);
};

template <typename Real, int DIR, int TL, int NL, int NT, int MINB, bool FINAL>
__global__ void __launch_bounds__(NT, MINB) sweep_kernel(SweepArgs<Real> a)
{
    using M = TileMap<DIR, TL, NL>;
    using S = SweepSmem<Real, TL, NL>;
    if (!a.ctl->active) return;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    Real *s_cell = reinterpret_cast<Real *>(smem_raw);  // [4][CELLS]
    Real *s_slope = s_cell + 4 * S::CELLS;              // [4][SLOPES]
    Real *s_flux = s_slope + 4 * S::SLOPES;             // [4][FLUXES]

    const int L = DIR == 0 ? a.nx : a.ny;
    const int NC = DIR == 0 ? a.ny : a.nx;
    const int tile = DIR == 0 ? blockIdx.x : blockIdx.y;
    const int ntiles = DIR == 0 ? gridDim.x : gridDim.y;
    const int l0 = 2 + tile * (TL - 1);
    const int c0 = (DIR == 0 ? blockIdx.y : blockIdx.x) * NL;
    const int fn = DIR == 0 ? 2 : 3;  // plane of the normal velocity
    const int ft = DIR == 0 ? 3 : 2;  // plane of the tangential velocity

    const double dt = a.ctl->dt;
    const Real h = Real(a.h), rh = Real(a.rh), alpha = Real(a.alpha), g = Real(a.gamma);
    const Real k = Real(dt);
    const Real lambda = Real(dt / a.h);

    auto gx = [&](int l, int c) { return DIR == 0 ? l : c0 + c; };
    auto gy = [&](int l, int c) { return DIR == 0 ? c0 + c : a.ny - 1 - l; };

    // 1. stage cells [l0-2, l0+TL] of NL lines
    for (int w = threadIdx.x; w < S::CELLS; w += NT) {
        int p, c;
        M::split(w, TL + 3, p, c);
        const int l = l0 - 2 + p;
        const int s = M::idx(p, c, TL + 3);
        if (l < L && c0 + c < NC) {
            const int x = gx(l, c), y = gy(l, c);
            s_cell[0 * S::CELLS + s] = a.src.at(0, x, y);
            s_cell[1 * S::CELLS + s] = a.src.at(1, x, y);
            s_cell[2 * S::CELLS + s] = a.src.at(fn, x, y);
            s_cell[3 * S::CELLS + s] = a.src.at(ft, x, y);
        } else {
            s_cell[0 * S::CELLS + s] = Real(1);
            s_cell[1 * S::CELLS + s] = Real(1);
            s_cell[2 * S::CELLS + s] = Real(0);
            s_cell[3 * S::CELLS + s] = Real(0);
        }
    }
    __syncthreads();

    // 2. limited slopes of cells l0-1+q, q in [0, TL]  (src/basicFuns.cuh:37-68)
    for (int w = threadIdx.x; w < S::SLOPES; w += NT) {
        int q, c;
        M::split(w, TL + 1, q, c);
        const int sm = M::idx(q, c, TL + 3), s0 = M::idx(q + 1, c, TL + 3), sp = M::idx(q + 2, c, TL + 3);
        const int d = M::idx(q, c, TL + 1);
#pragma unroll
        for (int f = 0; f < 4; ++f)
            s_slope[f * S::SLOPES + d] = limited_slope(s_cell[f * S::CELLS + sm], s_cell[f * S::CELLS + s0],
                                                       s_cell[f * S::CELLS + sp], rh, alpha);
    }
    __syncthreads();

    // 3. one relaxation GRP + midpoint flux per interface l-1/2, l = l0+i
    //    (src/basicFuns.cuh:75-192, 14-34)
    for (int w = threadIdx.x; w < S::FLUXES; w += NT) {
        int i, c;
        M::split(w, TL, i, c);
        const int l = l0 + i;
        const int d = M::idx(i, c, TL);
        Cell<Real> F = {Real(0), Real(0), Real(0), Real(0)};
        if (l <= L - 2 && c0 + c < NC) {
            const int sl = M::idx(i + 1, c, TL + 3), sr = M::idx(i + 2, c, TL + 3);
            const int ql = M::idx(i, c, TL + 1), qr = M::idx(i + 1, c, TL + 1);
            Cell<Real> sL, sR, fL, fR;
            sL.rho = s_slope[0 * S::SLOPES + ql]; sL.p = s_slope[1 * S::SLOPES + ql];
            sL.un = s_slope[2 * S::SLOPES + ql]; sL.ut = s_slope[3 * S::SLOPES + ql];
            sR.rho = s_slope[0 * S::SLOPES + qr]; sR.p = s_slope[1 * S::SLOPES + qr];
            sR.un = s_slope[2 * S::SLOPES + qr]; sR.ut = s_slope[3 * S::SLOPES + qr];
            // face states U -/+ s h / 2 (src/basicFuns.cuh:69-70)
            fL.rho = s_cell[0 * S::CELLS + sl] + sL.rho * h * Real(0.5);
            fL.p = s_cell[1 * S::CELLS + sl] + sL.p * h * Real(0.5);
            fL.un = s_cell[2 * S::CELLS + sl] + sL.un * h * Real(0.5);
            fL.ut = s_cell[3 * S::CELLS + sl] + sL.ut * h * Real(0.5);
            fR.rho = s_cell[0 * S::CELLS + sr] - sR.rho * h * Real(0.5);
            fR.p = s_cell[1 * S::CELLS + sr] - sR.p * h * Real(0.5);
            fR.un = s_cell[2 * S::CELLS + sr] - sR.un * h * Real(0.5);
            fR.ut = s_cell[3 * S::CELLS + sr] - sR.ut * h * Real(0.5);
            const Interface<Real> W = relaxation_grp(fL, fR, sL, sR, g);
            F = midpoint_flux(W, k);
        }
        s_flux[0 * S::FLUXES + d] = F.rho;
        s_flux[1 * S::FLUXES + d] = F.p;
        s_flux[2 * S::FLUXES + d] = F.un;
        s_flux[3 * S::FLUXES + d] = F.ut;
    }
    __syncthreads();

    // 4. conservative update of cells l0+i, i in [0, TL-1)  (src/basicFuns.cuh:229-246);
    //    ghost line positions 0,1 and L-2,L-1 pass through unchanged.
    double vmax = 0.0;
    auto emit = [&](int l, int c, const Cell<Real> &U) {
        const int x = gx(l, c), y = gy(l, c);
        if (FINAL) {
            // primitive average with branch A (src/basicFuns.cuh:264-274)
            const Real r = (a.comb.at(0, x, y) + U.rho) * Real(0.5);
            const Real p = (a.comb.at(1, x, y) + U.p) * Real(0.5);
            const Real u = (a.comb.at(fn, x, y) + U.un) * Real(0.5);
            const Real v = (a.comb.at(ft, x, y) + U.ut) * Real(0.5);
            a.dst.at(0, x, y) = r;
            a.dst.at(1, x, y) = p;
            a.dst.at(fn, x, y) = u;
            a.dst.at(ft, x, y) = v;
            if (x >= 2 && x <= a.nx - 3 && y >= 2 && y <= a.ny - 3)
                vmax = fmax(vmax, DIR == 0 ? wave_speed(r, p, u, v, a.gamma) : wave_speed(r, p, v, u, a.gamma));
        } else {
            a.dst.at(0, x, y) = U.rho;
            a.dst.at(1, x, y) = U.p;
            a.dst.at(fn, x, y) = U.un;
            a.dst.at(ft, x, y) = U.ut;
        }
    };
    for (int w = threadIdx.x; w < (TL - 1) * NL; w += NT) {
        int i, c;
        M::split(w, TL - 1, i, c);
        const int l = l0 + i;
        if (l > L - 3 || c0 + c >= NC) continue;
        const int s = M::idx(i + 2, c, TL + 3);
        Cell<Real> U;
        U.rho = s_cell[0 * S::CELLS + s]; U.p = s_cell[1 * S::CELLS + s];
        U.un = s_cell[2 * S::CELLS + s]; U.ut = s_cell[3 * S::CELLS + s];
        const int dl = M::idx(i, c, TL), dr = M::idx(i + 1, c, TL);
        Cell<Real> FL, FR;
        FL.rho = s_flux[0 * S::FLUXES + dl]; FL.p = s_flux[1 * S::FLUXES + dl];
        FL.un = s_flux[2 * S::FLUXES + dl]; FL.ut = s_flux[3 * S::FLUXES + dl];
        FR.rho = s_flux[0 * S::FLUXES + dr]; FR.p = s_flux[1 * S::FLUXES + dr];
        FR.un = s_flux[2 * S::FLUXES + dr]; FR.ut = s_flux[3 * S::FLUXES + dr];
        emit(l, c, conservative_update(U, FL, FR, lambda, g));
    }
    // pass-through lines (only the first and last tile hold them)
    if (tile == 0 || tile == ntiles - 1) {
        for (int w = threadIdx.x; w < 4 * NL; w += NT) {
            const int which = w / NL, c = w % NL;
            const int l = which < 2 ? which : L - 4 + which;  // 0, 1, L-2, L-1
            const int p = l - (l0 - 2);
            const bool mine = which < 2 ? (tile == 0) : (tile == ntiles - 1);
            if (!mine || p < 0 || p > TL + 2 || c0 + c >= NC) continue;
            const int s = M::idx(p, c, TL + 3);
            Cell<Real> U;
            U.rho = s_cell[0 * S::CELLS + s]; U.p = s_cell[1 * S::CELLS + s];
            U.un = s_cell[2 * S::CELLS + s]; U.ut = s_cell[3 * S::CELLS + s];
            emit(l, c, U);
        }
    }
    if (FINAL) block_max_to<NT>(vmax, &a.ctl->smax_bits);
}

// ---------------------------------------------------------------------------
// Ghost ring.  Presets are rows first, then columns (ghostCellPresets.cuh):
// the value a column rule copies from an interior column is that column's
// row-phase value, so each ring cell is computed directly from interior
// cells and no cell the kernel writes is read by it.
// ---------------------------------------------------------------------------
enum Strategy : int {
    OUTFLOW = 0,
    REFLECTIVE = 1,   // the reference runs its double-Mach kernel for it (wrappers.cuh:277-280)
    JET = 2,
    JET800 = 3,
    DOUBLE_MACH = 4,
    PERIODIC = 5,
    REFLECTIVE_TB = 6,
};

template <typename Real>
struct GhostArgs {
    Field<Real> U;
    int nx, ny, strategy;
    double gamma;
    StepControl *ctl;
    PlanParams plan;
};

template <typename Real>
__device__ __forceinline__ Cell<Real> load_prim(const Field<Real> &U, int x, int y)
{
    Cell<Real> c;
    c.rho = U.at(0, x, y); c.p = U.at(1, x, y); c.un = U.at(2, x, y); c.ut = U.at(3, x, y);
    return c;
}

template <typename Real>
__device__ __forceinline__ Cell<Real> mk(double r, double p, double u, double v)
{
    Cell<Real> c;
    c.rho = Real(r); c.p = Real(p); c.un = Real(u); c.ut = Real(v);
    return c;
}

// Row phase value of ring row j at column i (cells are (rho, p, u, v)).
template <typename Real>
__device__ __forceinline__ Cell<Real> row_rule(const GhostArgs<Real> &a, int i, int j, double t)
{
    const int ny = a.ny, nx = a.nx;
    Cell<Real> c;
    switch (a.strategy) {
    case OUTFLOW:
    case JET:  // ghostCellPresets.cuh:112-127, 156-171
        return load_prim(a.U, i, j < 2 ? 2 : ny - 3);
    case JET800:  // ghostCellPresets.cuh:204-219
        return load_prim(a.U, i, j < 2 ? 2 : (j == ny - 2 ? ny - 3 : ny - 4));
    case PERIODIC:  // wrap: 0<-ny-4, 1<-ny-3, ny-2<-2, ny-1<-3
        return load_prim(a.U, i, j == 0 ? ny - 4 : j == 1 ? ny - 3 : j == ny - 2 ? 2 : 3);
    case REFLECTIVE_TB:  // mirror with v negated: 0<-3, 1<-2, ny-2<-ny-3, ny-1<-ny-4
        c = load_prim(a.U, i, j == 0 ? 3 : j == 1 ? 2 : j == ny - 2 ? ny - 3 : ny - 4);
        c.ut = -c.ut;
        return c;
    default: {  // REFLECTIVE, DOUBLE_MACH: ghostCellPresets.cuh:56-92
        if (j == 0 || j == 1) {
            double temp = double(ny) / sqrt(3.0);
            double dist = double(ny) * 20 * t / sqrt(3.0);
            if (i <= nx / 24 + int(temp) + int(dist)) return mk<Real>(8, 116.5, 4.125 * sqrt(3.0), -4.125);
            return mk<Real>(1.4, 1, 0, 0);
        }
        if (j == ny - 1) {
            if (i <= nx / 24) return load_prim(a.U, i, j - 2);
            c = load_prim(a.U, i, j - 3);
            c.ut = -c.ut;
            return c;
        }
        c = load_prim(a.U, i, j - 1);
        if (i > nx / 24) c.ut = -c.ut;
        return c;
    }
    }
}

template <typename Real>
__device__ __forceinline__ bool ghost_row(int j, int ny) { return j < 2 || j >= ny - 2; }

// Row-phase state at (i, j): ring rows take their row rule, others are as is.
template <typename Real>
__device__ __forceinline__ Cell<Real> after_rows(const GhostArgs<Real> &a, int i, int j, double t)
{
    return ghost_row<Real>(j, a.ny) ? row_rule(a, i, j, t) : load_prim(a.U, i, j);
}

// Final value of ring column i at row j.
template <typename Real>
__device__ __forceinline__ Cell<Real> col_rule(const GhostArgs<Real> &a, int i, int j, double t)
{
    const int nx = a.nx, ny = a.ny;
    const bool left = i < 2;
    switch (a.strategy) {
    case OUTFLOW:
    case REFLECTIVE_TB:  // ghostCellPresets.cuh:129-144
        return after_rows(a, left ? 2 : nx - 3, j, t);
    case JET:  // ghostCellPresets.cuh:173-191
        if (left) {
            if (j >= 2 * ny / 5 + 1 && j <= 3 * ny / 5) return mk<Real>(5.0, 0.4127, 800.0, 0.0);
            return mk<Real>(0.5, 0.4127, 0.0, 0.0);
        }
        return after_rows(a, nx - 3, j, t);
    case JET800:  // ghostCellPresets.cuh:221-239
        if (left) {
            if (j >= 9 * ny / 10) return mk<Real>(1.4, 1, 800, 0);
            return mk<Real>(0.14, 1, 0, 0);
        }
        return after_rows(a, nx - 3, j, t);
    case PERIODIC:
        return after_rows(a, i == 0 ? nx - 4 : i == 1 ? nx - 3 : i == nx - 2 ? 2 : 3, j, t);
    default:  // ghostCellPresets.cuh:94-101
        if (left) return mk<Real>(8, 116.5, 4.125 * sqrt(3.0), -4.125);
        return mk<Real>(1.4, 1, 0, 0);
    }
}

// One thread per ring cell: 4 rows x nx, then 4 columns x (ny - 4).
template <typename Real, int NT>
__global__ void __launch_bounds__(NT) ghost_kernel(GhostArgs<Real> a)
{
    StepControl *ctl = a.ctl;
    if (!ctl->active) return;
    const double t = ctl->t + ctl->dt;  // the fill sees the advanced time (wrappers.cuh:250,265-280)
    const int nx = a.nx, ny = a.ny;
    const int nrow = 4 * nx, ncol = 4 * (ny - 4);
    const int k = blockIdx.x * NT + threadIdx.x;
    double vmax = 0.0;
    if (k < nrow + ncol) {
        int i, j;
        if (k < nrow) {
            const int r = k / nx;
            i = k % nx;
            j = r < 2 ? r : ny - 4 + r;
        } else {
            const int q = k - nrow;
            const int r = q / (ny - 4);
            j = 2 + q % (ny - 4);
            i = r < 2 ? r : nx - 4 + r;
        }
        const bool gcol = i < 2 || i >= nx - 2;
        const Cell<Real> c = gcol ? col_rule(a, i, j, t) : row_rule(a, i, j, t);
        a.U.at(0, i, j) = c.rho;
        a.U.at(1, i, j) = c.p;
        a.U.at(2, i, j) = c.un;
        a.U.at(3, i, j) = c.ut;
        vmax = wave_speed(c.rho, c.p, c.un, c.ut, a.gamma);
    }
    block_max_to<NT>(vmax, &ctl->smax_bits);
    if (last_block_done(&ctl->ticket)) {
        volatile StepControl *vc = ctl;
        ctl->t = vc->t + vc->dt;
        ctl->steps = vc->steps + 1;
        ctl->smax_last = __longlong_as_double((long long)vc->smax_bits);
        ctl->smax_bits = 0ull;
        ctl->ticket = 0u;
        plan_step(ctl, a.plan);
    }
}

} // namespace FVM2D_VARIANT
} // namespace fvm2d
