// fvm2d_batch.cuh -- batched kernels: many independent problems of different
// sizes advance together, one launch per stage of the step.
//
// Each problem keeps its own state buffers, step-control record (its own dt,
// time and end time) and ghost preset.  The work items of a stage -- x-sweep
// row segments, y-sweep column segments, ghost-ring blocks, init blocks -- of
// all problems form one list; prefix counts per problem map an item back to
// its problem.  Sweep items are dealt to warps in contiguous chunks (a warp
// meets few problem boundaries, so the final sweep folds its wave-speed max
// into a problem's record once per boundary).  Items of problems whose loop has
// ended are skipped.  The per-item arithmetic is the single-problem kernels'
// (x_item, y_item, ghost_cell).  In the contraction-free build a problem
// advanced in a batch matches the same problem advanced alone bit for bit; in
// the builds with FMA contraction the compiler may contract the inlined copies
// of that arithmetic differently in the two kernels, and the two agree to
// rounding.
#pragma once

#include "fvm2d_batch_control.h"
#include "fvm2d_kernels.cuh"

namespace fvm2d {
namespace FVM2D_VARIANT {

template <typename Real>
struct BatchArgs {
    Real *base;                // the batch allocation; problem buffers are element offsets into it
    const BatchProblem *prob;  // [np]
    StepControl *ctl;          // [np]
    const long long *x0;       // [np + 1] first x-sweep item of each problem
    const long long *y0;       // [np + 1] first y-sweep item of each problem
    const int *rb0;            // [np + 1] first ghost block of each problem
    const int *ib0;            // [np + 1] first init block of each problem
    int np;
};

// Largest p with first[p] <= item (first[] ascending, first[0] = 0).
template <typename T>
__device__ __forceinline__ int find_problem(const T *first, int np, T item)
{
    int lo = 0, hi = np - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (first[mid] <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// stage 0: X(U) -> A; 1: Y(U) -> B; 2: Y(A) -> U; 3: X(B) averaged with U -> U
template <typename Real>
__device__ __forceinline__ SweepArgs<Real> batch_sweep_args(const BatchArgs<Real> &b, int p, int stage)
{
    const BatchProblem &P = b.prob[p];
    const long long src = stage <= 1 ? P.u : (stage == 2 ? P.a : P.b);
    const long long dst = stage == 0 ? P.a : (stage == 1 ? P.b : P.u);
    SweepArgs<Real> a;
    a.src.base = b.base + src;
    a.dst.base = b.base + dst;
    a.comb.base = b.base + P.u;
    a.src.plane = a.dst.plane = a.comb.plane = P.plane;
    a.src.pitch = a.dst.pitch = a.comb.pitch = P.pitch;
    a.nx = P.nx;
    a.ny = P.ny;
    const bool x = (stage == 0 || stage == 3);
    a.h = x ? P.hx : P.hy;
    a.rh = x ? P.rhx : P.rhy;
    a.alpha = P.alpha;
    a.gamma = P.gamma;
    a.ctl = b.ctl + p;
    a.xchunks = P.xchunks;
    a.flux.base = nullptr;  // batches do not tape
    a.flux.plane = P.plane;
    a.flux.pitch = P.pitch;
    return a;
}

// Warp-wide max folded into *bits by lane 0 (values that are NaN never win).
__device__ __forceinline__ void warp_max_to(double v, unsigned long long *bits)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0 && v > 0.0) atomicMax(bits, (unsigned long long)__double_as_longlong(v));
}

template <typename Real, class Phys, bool FINAL, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) batch_sweep_x_kernel(BatchArgs<Real> b, long long total, int stage)
{
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (NT / 32);
    const long long wid = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32;
    const long long chunk = (total + nwarps - 1) / nwarps;
    long long it = wid * chunk;
    const long long end = min(it + chunk, total);
    int p = -1;
    long long pend = 0;
    bool active = false;
    double vmax = 0.0;
    int bad = 0;
    for (; it < end; ++it) {
        if (it >= pend) {
            if (FINAL && active) {
                note_bad_cells(bad, b.ctl + p);
                warp_max_to(vmax, &b.ctl[p].smax_bits);
            }
            vmax = 0.0;
            bad = 0;
            p = find_problem(b.x0, b.np, it);
            pend = b.x0[p + 1];
            active = b.ctl[p].active != 0;
            if (!active) {
                it = pend - 1;  // the loop of this problem has ended: skip its items
                continue;
            }
        }
        // the problem's arguments are re-read per item (cached loads), so none
        // of them is carried in registers across items
        const SweepArgs<Real> a = batch_sweep_args(b, p, stage);
        const SweepConsts<Real> K = sweep_consts(a, b.ctl[p].dt);
        const int nseg = b.prob[p].nsegx;
        const long long local = it - b.x0[p];
        x_item<Real, Phys, FINAL>(a, K, int(local / nseg), int(local % nseg), nseg, lane, vmax, bad);
    }
    if (FINAL && active) {
        note_bad_cells(bad, b.ctl + p);
        warp_max_to(vmax, &b.ctl[p].smax_bits);
    }
}

template <typename Real, class Phys, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB) batch_sweep_y_kernel(BatchArgs<Real> b, long long total, int stage)
{
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (NT / 32);
    const long long wid = (long long)blockIdx.x * (NT / 32) + threadIdx.x / 32;
    const long long chunk = (total + nwarps - 1) / nwarps;
    long long it = wid * chunk;
    const long long end = min(it + chunk, total);
    int p = -1;
    long long pend = 0;
    for (; it < end; ++it) {
        if (it >= pend) {
            p = find_problem(b.y0, b.np, it);
            pend = b.y0[p + 1];
            if (!b.ctl[p].active) {
                it = pend - 1;
                continue;
            }
        }
        const SweepArgs<Real> a = batch_sweep_args(b, p, stage);
        const SweepConsts<Real> K = sweep_consts(a, b.ctl[p].dt);
        const BatchProblem &P = b.prob[p];
        const long long local = it - b.y0[p];
        y_item<Real, Phys>(a, K, int(local / P.ncw), P.nsegy, int(local % P.ncw), lane, P.T);
    }
}

// True in one thread of the last of `nblocks` blocks to arrive at *ticket.
__device__ __forceinline__ bool last_of_blocks(unsigned int *ticket, unsigned int nblocks)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = (atomicAdd(ticket, 1u) == nblocks - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        return true;
    }
    return false;
}

template <typename Real, int NT>
__global__ void __launch_bounds__(NT) batch_ghost_kernel(BatchArgs<Real> b)
{
    const int p = find_problem(b.rb0, b.np, int(blockIdx.x));
    StepControl *ctl = b.ctl + p;
    if (!ctl->active) return;  // uniform over the block
    const BatchProblem &P = b.prob[p];
    GhostArgs<Real> g;
    g.U.base = b.base + P.u;
    g.U.plane = P.plane;
    g.U.pitch = P.pitch;
    g.nx = P.nx;
    g.ny = P.ny;
    g.strategy = P.strategy;
    g.gamma = P.gamma;
    g.ctl = ctl;
    g.plan = P.plan;
    g.row0 = 0;
    g.gny = P.ny;
    g.fill_top = g.fill_bottom = 1;
    const double t = ctl->t + ctl->dt;
    const int k = (int(blockIdx.x) - b.rb0[p]) * NT + threadIdx.x;
    const double v = (k < P.ring) ? ghost_cell(g, k, t) : 0.0;
    block_max_to<NT>(v, &ctl->smax_bits);
    if (last_of_blocks(&ctl->ticket, unsigned(b.rb0[p + 1] - b.rb0[p]))) finish_step(ctl, P.plan);
}

// Wave speed of every cell of each problem's initial state, then its first plan.
template <typename Real, int NT>
__global__ void __launch_bounds__(NT) batch_init_kernel(BatchArgs<Real> b)
{
    const int p = find_problem(b.ib0, b.np, int(blockIdx.x));
    const BatchProblem &P = b.prob[p];
    StepControl *ctl = b.ctl + p;
    Field<Real> U;
    U.base = b.base + P.u;
    U.plane = P.plane;
    U.pitch = P.pitch;
    const long long n = (long long)P.nx * P.ny;
    const long long first = (long long)(int(blockIdx.x) - b.ib0[p]) * kBatchInitCells;
    const long long last = min(first + kBatchInitCells, n);
    double m = 0.0;
    for (long long k = first + threadIdx.x; k < last; k += NT) {
        const int y = int(k / P.nx), x = int(k % P.nx);
        m = fmax(m, wave_speed(U.at(0, x, y), U.at(1, x, y), U.at(2, x, y), U.at(3, x, y), P.gamma));
    }
    block_max_to<NT>(m, &ctl->smax_bits);
    if (last_of_blocks(&ctl->ticket, unsigned(b.ib0[p + 1] - b.ib0[p]))) {
        volatile StepControl *vc = ctl;
        ctl->smax_last = __longlong_as_double((long long)vc->smax_bits);
        ctl->smax_bits = 0ull;
        ctl->ticket = 0u;
        plan_step(ctl, P.plan);
    }
}

template <typename Real>
__global__ void batch_plan_kernel(BatchArgs<Real> b)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < b.np) plan_step(b.ctl + p, b.prob[p].plan);
}

} // namespace FVM2D_VARIANT
} // namespace fvm2d
