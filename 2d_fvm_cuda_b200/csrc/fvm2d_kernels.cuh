// fvm2d_kernels.cuh -- the sm_100a kernels of one split step.
//
// A step is  U <- ghost( (Y(X(U)) + X(Y(U))) / 2 )  with one dt
// (src/wrappers.cuh:196-284).  It runs as five kernels, all reading the step
// size from a device-resident control record so the loop never waits on the
// host:
//
//   sweep_x        U -> A         first sweep of branch A
//   sweep_y        U -> B         first sweep of branch B
//   sweep_y        A -> U         second sweep of branch A (U^n is dead now)
//   sweep_x final  B -> U         second sweep of branch B, fused with the
//                                 primitive average against U (branch A) and
//                                 the wave-speed max of the interior cells
//   ghost_kernel   U -> U         boundary ring for the preset, wave-speed
//                                 max of the ring, and (last block) the time
//                                 advance plus the next step's dt
//
// Every limited slope, interface (relaxation GRP + midpoint flux) and cell
// update lives in registers; the reference's slope, face-state, interface
// and transposed buffers never reach HBM.  The y-sweep indexes rows in
// reverse (line position l = ny-1-j) with (un, ut) = (v, u), which is the
// reference's anti-transpose (src/basicFuns.cuh:249-262) applied in the
// indexing instead of through global memory.
#pragma once

#include "fvm2d_control.h"
#include "fvm2d_math.cuh"
#include "fvm2d_split.cuh"

#include <stdint.h>
#include <type_traits>

namespace fvm2d {
namespace FVM2D_VARIANT {

// Start the next step if the loop of wrappers.cuh:196-207 continues:
// dt = min(CFL h / smax, t_end - t); stop when t >= t_end or h/smax < 1e-20.
// With a fixed step size (differentiation runs) dt is that constant and only
// the step limit ends the loop.
__device__ __forceinline__ void plan_step(StepControl *c, const PlanParams &p)
{
    c->active = 0;
    if (c->done) return;
    if (c->steps >= c->step_limit) return;
    if (p.fixed_dt > 0.0) {  // differentiation runs: a constant step size, bounded by the step count only
        c->dt = p.fixed_dt;
        c->active = 1;
        return;
    }
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

// A row slab of a problem split across devices plans its step from the
// wave-speed maximum over all slabs, which the caller's reduction left in
// device memory, so no slab waits on the host between steps.
__global__ void plan_from_kernel(StepControl *c, PlanParams p, const double *smax)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        c->smax_last = *smax;
        plan_step(c, p);
    }
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

// Records the step in flight as the first to leave a bad cell, if any lane of
// the warp saw one and no earlier step did.  Called by all lanes of a warp.
__device__ __forceinline__ void note_bad_cells(int bad, StepControl *ctl)
{
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicCAS(&ctl->first_bad, 0, ctl->steps + 1);
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
        // single precision: 32-bit in-plane offsets (pitch * ny < 2^31 is
        // checked when a solver or batch is created), measured 5% faster on
        // the issue-bound FP32 sweeps; no faster in FP64
        if constexpr (sizeof(Real) == 4) return base[(long long)f * plane + (y * pitch + x)];
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
    int xchunks;       // x-sweeps: chunks of 32 cells per work item (fvm2d_control.h)
    Field<Real> flux;  // taped sweeps only (base null otherwise): each interface's flux (planes:
                       // mass, normal momentum, energy, tangential momentum) at the interface's right cell
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
// Sweep kernels.  Neither uses shared memory or a block barrier: every warp
// works on its own pieces of the array, so a warp waiting on FP64 latency
// never holds others back.  Both walk the array with a grid-stride loop over
// work items; the grid is sized to the kernel's occupancy.
//
// x-sweep: a work item is a segment of one row, walked by a warp in chunks
// of 32 consecutive cells.  In a chunk lane k holds cell c: it loads cells
// c-1..c+1 (coalesced), computes the limited slope of c, takes the slope of
// c-1 from lane k-1 by shuffle and computes the interface c-1/2, then takes
// the flux of c-3/2 from lane k-1 and updates cell c-1.  Lane 0 takes the
// slope and flux it needs from lane 31 of the previous chunk, so after the
// first chunk every lane of every chunk does useful work (in the first chunk
// lanes 0 and 1 only feed their neighbours).
//
// y-sweep: a work item is 32 consecutive columns times one segment of T
// interfaces along y.  Each lane walks its column in line order (line
// position l = ny-1-j, so the "left" cell of an interface is the one below
// it, as in the reference's anti-transposed copy) keeping three cells, the
// last slope and the last flux in registers: one cell load (issued one
// iteration before its use), one slope, one interface and one update per
// iteration.  Loads and stores of a
// warp touch 32 consecutive doubles of a row.
// ---------------------------------------------------------------------------
template <typename Real>
__device__ __forceinline__ SweepConsts<Real> sweep_consts(const SweepArgs<Real> &a, double dt)
{
    SweepConsts<Real> K;
    K.h = Real(a.h);
    K.rh = Real(a.rh);
    K.alpha = Real(a.alpha);
    set_gamma_consts(K, a.gamma);
    K.k = Real(dt);
    K.lambda = Real(dt / a.h);
    K.lambda_lo = Real(lo_part<Real>(dt / a.h));
    return K;
}

template <typename Real>
__device__ __forceinline__ Cell<Real> load_cell(const Field<Real> &F, int x, int y, int fn, int ft)
{
    Cell<Real> c;
    c.rho = F.at(0, x, y);
    c.p = F.at(1, x, y);
    c.un = F.at(fn, x, y);
    c.ut = F.at(ft, x, y);
    return c;
}

template <typename Real>
__device__ __forceinline__ void store_cell(const Field<Real> &F, int x, int y, int fn, int ft, const Cell<Real> &c)
{
    F.at(0, x, y) = c.rho;
    F.at(1, x, y) = c.p;
    F.at(fn, x, y) = c.un;
    F.at(ft, x, y) = c.ut;
}

// ---- FP32 states with residual planes -------------------------------------
// A stored value is the FP32 plane value plus its plane's 16-bit residual
// (fvm2d_split.cuh).  With a physics that declares kSplitStorage (and
// provides update_split), the sweeps read the FP32 values for slopes and
// fluxes and hi + lo of the cell they update, and write the result split
// again.
template <class P, class = void>
struct split_storage : std::false_type {};
template <class P>
struct split_storage<P, std::void_t<decltype(P::kSplitStorage)>> : std::integral_constant<bool, P::kSplitStorage> {};

// the 8-byte word of a cell's 4 residuals (field f in bits 16 f .. 16 f + 15)
template <typename Real>
__device__ __forceinline__ unsigned long long &lo_cell(const Field<Real> &F, int x, int y)
{
    return reinterpret_cast<unsigned long long *>(residual_block(F.base, F.plane))[y * F.pitch + x];
}

// the residuals of a cell, as values of the arithmetic type
template <typename Real>
__device__ __forceinline__ Cell<Real> load_lo(const Field<Real> &F, int x, int y, int fn, int ft)
{
    const unsigned long long w = lo_cell(F, x, y);
    auto part = [&](int f) { return Real(bf16_value((unsigned short)(w >> (16 * f)))); };
    Cell<Real> c;
    c.rho = part(0);
    c.p = part(1);
    c.un = part(fn);
    c.ut = part(ft);
    return c;
}

template <typename Real>
__device__ __forceinline__ Cell<double> join_cell(const Cell<Real> &hi, const Cell<Real> &lo)
{
    return {double(hi.rho) + double(lo.rho), double(hi.p) + double(lo.p), double(hi.un) + double(lo.un),
            double(hi.ut) + double(lo.ut)};
}

// v split into the FP32 planes and the cell's residual word; returns the
// FP32 part
template <typename Real>
__device__ __forceinline__ Cell<Real> store_split(const Field<Real> &F, int x, int y, int fn, int ft,
                                                  const Cell<double> &v)
{
    float h[4];
    unsigned short l[4];
    split_value(v.rho, h[0], l[0]);
    split_value(v.p, h[1], l[1]);
    split_value(v.un, h[2], l[fn]);
    split_value(v.ut, h[3], l[ft]);
    lo_cell(F, x, y) = (unsigned long long)l[0] | (unsigned long long)l[1] << 16 | (unsigned long long)l[2] << 32 |
                       (unsigned long long)l[3] << 48;
    const Cell<Real> hi = {Real(h[0]), Real(h[1]), Real(h[2]), Real(h[3])};
    store_cell(F, x, y, fn, ft, hi);
    return hi;
}

// a cell's residuals copied (ghost cells passing through a sweep)
template <typename Real>
__device__ __forceinline__ void copy_lo(const Field<Real> &from, const Field<Real> &to, int x, int y)
{
    lo_cell(to, x, y) = lo_cell(from, x, y);
}

// Value of the next (lane_down) or previous (lane_up) lane of the warp, or of
// its last lane (lane_last).
__device__ __forceinline__ double lane_down(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float lane_down(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double lane_up(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float lane_up(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double lane_last(double v) { return __shfl_sync(0xffffffffu, v, 31); }
__device__ __forceinline__ float lane_last(float v) { return __shfl_sync(0xffffffffu, v, 31); }

template <typename Real>
__device__ __forceinline__ Cell<Real> shfl_down(const Cell<Real> &c)
{
    Cell<Real> o;
    o.rho = lane_down(c.rho);
    o.p = lane_down(c.p);
    o.un = lane_down(c.un);
    o.ut = lane_down(c.ut);
    return o;
}

template <typename Real>
__device__ __forceinline__ Cell<Real> shfl_up(const Cell<Real> &c)
{
    Cell<Real> o;
    o.rho = lane_up(c.rho);
    o.p = lane_up(c.p);
    o.un = lane_up(c.un);
    o.ut = lane_up(c.ut);
    return o;
}

template <typename Real>
__device__ __forceinline__ Cell<Real> shfl_last(const Cell<Real> &c)
{
    Cell<Real> o;
    o.rho = lane_last(c.rho);
    o.p = lane_last(c.p);
    o.un = lane_last(c.un);
    o.ut = lane_last(c.ut);
    return o;
}

// Asynchronous global->shared copies of single elements (cp.async groups,
// waited for by the issuing thread).
template <typename Real>
__device__ __forceinline__ void async_copy(Real *dst_shared, const Real *src)
{
#if defined(__CUDA_ARCH__)
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst_shared);
    if constexpr (sizeof(Real) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(src) : "memory");
#else
    *dst_shared = *src;  // host builds of this file (tests): a plain copy
#endif
}
__device__ __forceinline__ void async_commit()
{
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.commit_group;" ::: "memory");
#endif
}
template <int N>
__device__ __forceinline__ void async_wait()
{
#if defined(__CUDA_ARCH__)
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
#endif
}

// An x-sweep work item of a.xchunks chunks of 32 cells: item seg starts at
// cell b0 = 1 + cells seg (lane 0 of its first chunk) and updates cells
// b0+1 .. b0+cells, cells = 32 xchunks - 2 (fvm2d_control.h).

// One x-sweep work item: row y, segment seg (of nseg).  vmax collects the
// wave speed of the interior cells written by a final sweep, and bad whether
// one of them holds NaN or a non-positive density or pressure; a taped sweep
// also stores every interface flux it computes.
//
// RING = D > 0: the warp streams its row through a ring of kXRingChunks
// chunk slots in shared memory (`ring`: this warp's slots, 4 fields of 32
// cells each), filled by asynchronous copies D chunks ahead of use; a lane
// reads its three cells there instead of from global memory.
constexpr int kXRingChunks = 8;
// prefetch distance (chunks) of the first x-sweep's ring; 0: no ring
#ifndef FVM2D_X_RING
#define FVM2D_X_RING 4
#endif

template <typename Real, class Phys, bool FINAL, int RING = 0>
__device__ __forceinline__ void x_item(const SweepArgs<Real> &a, const SweepConsts<Real> &K, int y, int seg,
                                       int nseg, int lane, double &vmax, int &bad, Real *ring = nullptr)
{
    const int nx = a.nx, ny = a.ny;
    // a taped sweep (a.flux set) stores every interface flux; the same code
    // runs taped and untaped, so both give the same bits
    const bool tape = a.flux.base != nullptr;
    constexpr bool kResidual = split_storage<Phys>::value;
    const int cells = x_item_cells(a.xchunks);
    const int b0 = 1 + seg * cells;
    const int last = min(b0 + cells, nx - 3);  // last cell this item updates
    auto ld = [&](int x) { return load_cell(a.src, min(max(x, 0), nx - 1), y, 2, 3); };
    auto emit = [&](int x, const Cell<Real> &U, const Cell<Real> &Ab) {
        if (FINAL) {
            Cell<Real> o;  // primitive average with branch A (src/basicFuns.cuh:264-274)
            o.rho = (Ab.rho + U.rho) * Real(0.5);
            o.p = (Ab.p + U.p) * Real(0.5);
            o.un = (Ab.un + U.un) * Real(0.5);
            o.ut = (Ab.ut + U.ut) * Real(0.5);
            store_cell(a.dst, x, y, 2, 3, o);
            if (x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3) {
                vmax = fmax(vmax, wave_speed(o.rho, o.p, o.un, o.ut, a.gamma));
                bad |= !(o.rho > Real(0) && o.p > Real(0));  // NaN fails both tests
            }
        } else {
            store_cell(a.dst, x, y, 2, 3, U);
        }
    };
    // residual builds: U and Ab as hi + lo; the wave speed from the FP32 part
    // as stored (as the init and ghost kernels see it)
    auto emit_split = [&](int x, const Cell<double> &U, const Cell<double> &Ab) {
        if (FINAL) {
            const Cell<double> o = {(Ab.rho + U.rho) * 0.5, (Ab.p + U.p) * 0.5, (Ab.un + U.un) * 0.5,
                                    (Ab.ut + U.ut) * 0.5};
            const Cell<Real> h = store_split(a.dst, x, y, 2, 3, o);
            if (x >= 2 && x <= nx - 3 && y >= 2 && y <= ny - 3) {
                vmax = fmax(vmax, wave_speed(h.rho, h.p, h.un, h.ut, a.gamma));
                bad |= !(h.rho > Real(0) && h.p > Real(0));
            }
        } else {
            store_split(a.dst, x, y, 2, 3, U);
        }
    };
    // chunk m's cell of this lane into its ring slot
    auto issue = [&](int m) {
        const int x = min(max(b0 + 32 * m + lane, 0), nx - 1);
        Real *r = ring + (m & (kXRingChunks - 1)) * 128 + lane;
        async_copy(r, &a.src.at(0, x, y));
        async_copy(r + 32, &a.src.at(1, x, y));
        async_copy(r + 64, &a.src.at(2, x, y));
        async_copy(r + 96, &a.src.at(3, x, y));
    };
    auto get = [&](int m, int k) {
        const Real *r = ring + (m & (kXRingChunks - 1)) * 128 + k;
        Cell<Real> q;
        q.rho = r[0];
        q.p = r[32];
        q.un = r[64];
        q.ut = r[96];
        return q;
    };
    if constexpr (RING > 0) {
        static_assert(RING + 3 <= kXRingChunks, "prefetch distance does not fit the ring");
        issue(0);
        issue(1);
        async_commit();
        for (int m = 2; m <= RING; ++m) {
            issue(m);
            async_commit();
        }
    }
    Cell<Real> cs = {Real(0), Real(0), Real(0), Real(0)}, cF = cs;  // lane 31's slope and flux, previous chunk
    for (int j = 0; j < a.xchunks; ++j) {
        const int b = b0 + 32 * j;
        if (b - 1 > last) break;  // nothing left to update (the same for the whole warp)
        const int c = b + lane, u = c - 1;  // this lane's cell, and the cell it updates
        Cell<Real> cm1, c0, cp1;
        if constexpr (RING > 0) {
            issue(j + RING + 1);
            async_commit();
            async_wait<RING>();  // chunks up to j+1 have landed (this lane's copies)
            __syncwarp();        // ... and every lane's
            cm1 = lane > 0 ? get(j, lane - 1) : (j > 0 ? get(j - 1, 31) : ld(c - 1));
            c0 = get(j, lane);
            cp1 = lane < 31 ? get(j, lane + 1) : get(j + 1, 0);
        } else {
            cm1 = ld(c - 1);
            c0 = ld(c);
            cp1 = ld(c + 1);
        }
        Cell<Real> A, Alo, Ulo;
        if (FINAL) A = load_cell(a.comb, min(max(u, 0), nx - 1), y, 2, 3);  // branch A, loaded early
        if (FINAL && kResidual) Alo = load_lo(a.comb, min(max(u, 0), nx - 1), y, 2, 3);
        if (kResidual) Ulo = load_lo(a.src, min(max(u, 0), nx - 1), y, 2, 3);  // the updated cell's, early
        const Cell<Real> s0 = Phys::slope(cm1, c0, cp1, K);                // slope of cell c
        Cell<Real> sm1 = shfl_up(s0);                                     // slope of cell c-1
        if (lane == 0) sm1 = cs;
        Cell<Real> F = {Real(0), Real(0), Real(0), Real(0)};
        if (c <= nx - 2) F = Phys::interface_flux(cm1, c0, sm1, s0, K);   // interface c-1/2
        if (tape && (j > 0 || lane >= 1) && c <= nx - 2) store_cell(a.flux, c, y, 2, 3, F);  // at cell c
        Cell<Real> FL = shfl_up(F);                                       // interface c-3/2
        if (lane == 0) FL = cF;
        if ((j > 0 || lane >= 2) && u <= last) {
            if constexpr (kResidual)
                emit_split(u, Phys::update_split(cm1, Ulo, FL, F, K), join_cell(A, Alo));
            else
                emit(u, Phys::update(cm1, FL, F, K), A);
        }
        cs = shfl_last(s0);
        cF = shfl_last(F);
    }
    if constexpr (RING > 0) {
        async_wait<0>();  // no copy of this item may land in the ring after it
        __syncwarp();
    }
    // ghost columns pass through (x-sweeps do not update them, src/basicFuns.cuh:235)
    auto pass = [&](int x) {
        Cell<Real> Ab;
        if (FINAL) Ab = load_cell(a.comb, x, y, 2, 3);
        if constexpr (kResidual) {
            Cell<Real> Ablo;
            if (FINAL) Ablo = load_lo(a.comb, x, y, 2, 3);
            emit_split(x, join_cell(ld(x), load_lo(a.src, x, y, 2, 3)), join_cell(Ab, Ablo));
        } else {
            emit(x, ld(x), Ab);
        }
    };
    if (lane < 2 && (seg == 0 || seg == nseg - 1)) {
        pass(seg == 0 ? lane : nx - 2 + lane);
        if (seg == 0 && seg == nseg - 1) pass(nx - 2 + lane);
    }
}

template <typename Real, class Phys, bool FINAL, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) sweep_x_kernel(SweepArgs<Real> a)
{
    if (!a.ctl->active) return;
    const SweepConsts<Real> K = sweep_consts(a, a.ctl->dt);
    const int lane = threadIdx.x & 31;
    const int nseg = x_items_per_row(a.nx, a.xchunks);
    const long long nwork = (long long)nseg * a.ny;
    const long long wstride = (long long)gridDim.x * (NT / 32);
    double vmax = 0.0;
    int bad = 0;
    // the ring serves the first FP64 x-sweep; the final one (which also
    // reads branch A and reduces over the block) and the issue-bound FP32
    // ones were measured slower with it
    constexpr int RING = (!FINAL && sizeof(Real) == 8) ? FVM2D_X_RING : 0;
    if constexpr (RING > 0) {
        __shared__ Real ring[(NT / 32) * kXRingChunks * 128];
        Real *mine = ring + (threadIdx.x / 32) * kXRingChunks * 128;
        for (long long w = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32; w < nwork; w += wstride)
            x_item<Real, Phys, FINAL, RING>(a, K, int(w / nseg), int(w % nseg), nseg, lane, vmax, bad, mine);
    } else {
        for (long long w = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32; w < nwork; w += wstride)
            x_item<Real, Phys, FINAL>(a, K, int(w / nseg), int(w % nseg), nseg, lane, vmax, bad);
    }
    if (FINAL) {
        note_bad_cells(bad, a.ctl);
        block_max_to<NT>(vmax, &a.ctl->smax_bits);
    }
}

// Segments of T interfaces (T-1 updated cells) along a y line of ny cells.
__host__ __device__ __forceinline__ int y_segments(int ny, int T) { return (ny - 4 + T - 2) / (T - 1); }

// One y-sweep work item: columns 32 cw .. 32 cw + 31, segment seg (of nseg)
// of T interfaces.  A taped sweep also stores every interface flux.
//
// RING = 0: the walker keeps its three cells, the next one (loaded one
// interface ahead), the last slope and the last flux in registers.
// RING = D > 0: each lane streams its column through a ring of kYRingRows
// rows in shared memory (`ring`, rows of 4 fields, consecutive entries
// `rs` elements apart, one column per thread), filled by asynchronous
// global->shared copies issued D rows ahead of use and waited for per
// thread (cp.async groups: no barrier, no other thread involved); the
// registers then hold only the last slope and flux across the Riemann
// solver, and the loads never stall the walker.
constexpr int kYRingRows = 8;

template <typename Real, class Phys, int RING = 0>
__device__ __forceinline__ void y_item(const SweepArgs<Real> &a, const SweepConsts<Real> &K, int seg, int nseg,
                                       int cw, int lane, int T, Real *ring = nullptr, int rs = 0,
                                       unsigned long long *ring_lo = nullptr)
{
    const int nx = a.nx, ny = a.ny;
    const bool tape = a.flux.base != nullptr;  // as in x_item
    constexpr bool kResidual = split_storage<Phys>::value;
    const int x = cw * 32 + lane;
    const bool col = x < nx;
    const int xc = col ? x : nx - 1;
    const int l0 = 2 + seg * (T - 1);
    const int lend = min(l0 + T - 1, ny - 2);  // last interface of the segment
    auto ld = [&](int l) { return load_cell(a.src, xc, ny - 1 - l, 3, 2); };
    if constexpr (RING == 0) {
        Cell<Real> cm1 = ld(l0 - 1), c0 = ld(l0), cp1 = ld(l0 + 1);
        Cell<Real> sm1 = Phys::slope(ld(l0 - 2), cm1, c0, K);
        Cell<Real> Fp = {Real(0), Real(0), Real(0), Real(0)};
        for (int l = l0; l <= lend; ++l) {
            const Cell<Real> cp2 = ld(min(l + 2, ny - 1));  // next iteration's cell, loaded one interface ahead
            const Cell<Real> s0 = Phys::slope(cm1, c0, cp1, K);
            const Cell<Real> F = Phys::interface_flux(cm1, c0, sm1, s0, K);
            if (tape && col) store_cell(a.flux, x, ny - 1 - l, 2, 3, F);  // interface l-1/2 at line position l
            if (l > l0 && col) {  // cell l-1
                if constexpr (kResidual)
                    store_split(a.dst, x, ny - l, 3, 2, Phys::update_split(cm1, load_lo(a.src, x, ny - l, 3, 2), Fp, F, K));
                else
                    store_cell(a.dst, x, ny - l, 3, 2, Phys::update(cm1, Fp, F, K));
            }
            Fp = F;
            cm1 = c0;
            c0 = cp1;
            cp1 = cp2;
            sm1 = s0;
        }
    } else {
        static_assert(RING >= 1 && RING + 3 <= kYRingRows, "prefetch distance does not fit the ring");
        // row l of the line (clamped to the array) into its ring slot, fields (rho, p, un, ut)
        auto issue = [&](int l) {
            const int y = ny - 1 - min(l, ny - 1);
            Real *r = ring + (l & (kYRingRows - 1)) * 4 * rs;
            async_copy(r, &a.src.at(0, xc, y));
            async_copy(r + rs, &a.src.at(1, xc, y));
            async_copy(r + 2 * rs, &a.src.at(3, xc, y));
            async_copy(r + 3 * rs, &a.src.at(2, xc, y));
            // residual builds: the row's residual word rides in the ring too
            if constexpr (kResidual) async_copy(ring_lo + (l & (kYRingRows - 1)) * rs, &lo_cell(a.src, xc, y));
        };
        auto get_lo = [&](int l) {  // the residuals of row l, in (rho, p, un, ut) order
            const unsigned long long w = ring_lo[(l & (kYRingRows - 1)) * rs];
            auto part = [&](int f) { return Real(bf16_value((unsigned short)(w >> (16 * f)))); };
            return Cell<Real>{part(0), part(1), part(3), part(2)};
        };
        auto get = [&](int l) {
            const Real *r = ring + (l & (kYRingRows - 1)) * 4 * rs;
            Cell<Real> c;
            c.rho = r[0];
            c.p = r[rs];
            c.un = r[2 * rs];
            c.ut = r[3 * rs];
            return c;
        };
        for (int l = l0 - 2; l <= l0 + 1; ++l) issue(l);
        async_commit();
        for (int k = 1; k < RING; ++k) {  // rows l0+2 .. l0+RING, one group each
            issue(l0 + 1 + k);
            async_commit();
        }
        async_wait<RING - 1>();  // rows up to l0+1 have landed
        Cell<Real> sm1 = Phys::slope(get(l0 - 2), get(l0 - 1), get(l0), K);
        Cell<Real> Fp = {Real(0), Real(0), Real(0), Real(0)};
        for (int l = l0; l <= lend; ++l) {
            issue(l + RING + 1);  // RING rows ahead of the row this iteration needs last
            async_commit();
            async_wait<RING>();   // rows up to l+1 have landed
            const Cell<Real> cm1 = get(l - 1), c0 = get(l), cp1 = get(l + 1);
            const Cell<Real> s0 = Phys::slope(cm1, c0, cp1, K);
            const Cell<Real> F = Phys::interface_flux(cm1, c0, sm1, s0, K);
            if (tape && col) store_cell(a.flux, x, ny - 1 - l, 2, 3, F);
            if (l > l0 && col) {
                if constexpr (kResidual)
                    store_split(a.dst, x, ny - l, 3, 2, Phys::update_split(cm1, get_lo(l - 1), Fp, F, K));
                else
                    store_cell(a.dst, x, ny - l, 3, 2, Phys::update(get(l - 1), Fp, F, K));
            }
            Fp = F;
            sm1 = s0;
        }
        async_wait<0>();  // no copy of this item may land in the ring after it
    }
    // ghost rows pass through (y-sweeps do not update them)
    auto pass = [&](int l) {
        store_cell(a.dst, x, ny - 1 - l, 3, 2, ld(l));
        if constexpr (kResidual) copy_lo(a.src, a.dst, x, ny - 1 - l);
    };
    if (col && seg == 0)
        for (int l = 0; l < 2; ++l) pass(l);
    if (col && seg == nseg - 1)
        for (int l = ny - 2; l < ny; ++l) pass(l);
}

// prefetch distance of the y walker's shared-memory ring (rows; 0: no ring);
// measured at 4096^2: the ring makes the FP64 y-sweeps 21% faster (they no
// longer spill the walker's cells), the FP32 ones 4%
#ifndef FVM2D_Y_RING
#define FVM2D_Y_RING 4
#endif

template <typename Real, class Phys, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) sweep_y_kernel(SweepArgs<Real> a, int T)
{
    if (!a.ctl->active) return;
    const SweepConsts<Real> K = sweep_consts(a, a.ctl->dt);
    const int lane = threadIdx.x & 31;
    const int ncw = (a.nx + 31) / 32;
    const int nseg = y_segments(a.ny, T);
    const long long nwork = (long long)ncw * nseg;
    const long long wstride = (long long)gridDim.x * (NT / 32);
    constexpr int RING = (sizeof(Real) == 4 || sizeof(Real) == 8) ? FVM2D_Y_RING : 0;
    if constexpr (RING > 0 && split_storage<Phys>::value) {
        __shared__ Real ring[kYRingRows * 4 * NT];
        __shared__ unsigned long long ring_lo[kYRingRows * NT];
        for (long long w = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32; w < nwork; w += wstride)
            y_item<Real, Phys, RING>(a, K, int(w / ncw), nseg, int(w % ncw), lane, T, ring + threadIdx.x, NT,
                                     ring_lo + threadIdx.x);
    } else if constexpr (RING > 0) {
        __shared__ Real ring[kYRingRows * 4 * NT];
        for (long long w = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32; w < nwork; w += wstride)
            y_item<Real, Phys, RING>(a, K, int(w / ncw), nseg, int(w % ncw), lane, T, ring + threadIdx.x, NT);
    } else {
        for (long long w = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32; w < nwork; w += wstride)
            y_item<Real, Phys>(a, K, int(w / ncw), nseg, int(w % ncw), lane, T);
    }
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
    int row0, gny;               // global row of local row 0; global row count
    int fill_top, fill_bottom;   // 0: that pair of ring rows is a halo (not filled, no max)
    int residual = 0;            // 1: the state has residual planes (a ring cell's are zeroed)
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
            double temp = double(a.gny) / sqrt(3.0);
            double dist = double(a.gny) * 20 * t / sqrt(3.0);
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
    const int nx = a.nx;
    const bool left = i < 2;
    switch (a.strategy) {
    case OUTFLOW:
    case REFLECTIVE_TB:  // ghostCellPresets.cuh:129-144
        return after_rows(a, left ? 2 : nx - 3, j, t);
    case JET:  // ghostCellPresets.cuh:173-191
        if (left) {
            const int gj = a.row0 + j, gny = a.gny;
            if (gj >= 2 * gny / 5 + 1 && gj <= 3 * gny / 5) return mk<Real>(5.0, 0.4127, 800.0, 0.0);
            return mk<Real>(0.5, 0.4127, 0.0, 0.0);
        }
        return after_rows(a, nx - 3, j, t);
    case JET800:  // ghostCellPresets.cuh:221-239
        if (left) {
            if (a.row0 + j >= 9 * a.gny / 10) return mk<Real>(1.4, 1, 800, 0);
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

// Ring cell k of 4 nx + 4 (ny - 4): rows 0, 1, ny-2, ny-1 first, then
// columns 0, 1, nx-2, nx-1 of rows 2..ny-3.  Writes the cell and returns its
// wave speed.
template <typename Real>
__device__ __forceinline__ double ghost_cell(const GhostArgs<Real> &a, int k, double t)
{
    const int nx = a.nx, ny = a.ny;
    const int nrow = 4 * nx;
    int i, j;
    if (k < nrow) {
        const int r = k / nx;
        if (!(r < 2 ? a.fill_top : a.fill_bottom)) return 0.0;  // halo rows of a slab
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
    if (a.residual) lo_cell(a.U, i, j) = 0ull;  // a ring cell holds its FP32 value exactly
    return wave_speed(c.rho, c.p, c.un, c.ut, a.gamma);
}

// Commits the step in flight (t += dt, steps + 1), takes the running wave-speed
// max as the new state's, and plans the next step.  One thread, after every
// contribution to smax_bits is visible.
__device__ __forceinline__ void finish_step(StepControl *ctl, const PlanParams &plan)
{
    volatile StepControl *vc = ctl;
    ctl->t = vc->t + vc->dt;
    ctl->steps = vc->steps + 1;
    ctl->smax_last = __longlong_as_double((long long)vc->smax_bits);
    ctl->smax_bits = 0ull;
    ctl->ticket = 0u;
    plan_step(ctl, plan);
}

// One thread per ring cell.
template <typename Real, int NT>
__global__ void __launch_bounds__(NT) ghost_kernel(GhostArgs<Real> a)
{
    StepControl *ctl = a.ctl;
    if (!ctl->active) return;
    const double t = ctl->t + ctl->dt;  // the fill sees the advanced time (wrappers.cuh:250,265-280)
    const int k = blockIdx.x * NT + threadIdx.x;
    const double vmax = (k < 4 * a.nx + 4 * (a.ny - 4)) ? ghost_cell(a, k, t) : 0.0;
    block_max_to<NT>(vmax, &ctl->smax_bits);
    if (last_block_done(&ctl->ticket)) finish_step(ctl, a.plan);
}

} // namespace FVM2D_VARIANT
} // namespace fvm2d
