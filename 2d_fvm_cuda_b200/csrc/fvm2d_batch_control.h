// fvm2d_batch_control.h -- records shared by the batched kernels and the
// batch host runtime.
#pragma once

#include "fvm2d_control.h"

namespace fvm2d {

// Device descriptor of one problem of a batch.
struct BatchProblem {
    long long u, a, b;     // element offsets of the state and the two sweep buffers
    long long plane;       // elements between field planes
    int pitch, nx, ny, strategy;
    double hx, hy, rhx, rhy, alpha, gamma;
    PlanParams plan;
    int nsegx;             // x-sweep segments per row
    int ncw, nsegy, T;     // y-sweep: 32-column groups, segments per column, interfaces per segment
    int ring;              // ghost-ring cells
    int xchunks;           // x-sweep: chunks of 32 cells per work item (fvm2d_control.h)
};

// Cells per block of the batched initial wave-speed reduction.
constexpr int kBatchInitCells = 256 * 16;

// Everything one build of the kernels needs to enqueue a batched step.
struct BatchLaunch {
    void *base;
    const BatchProblem *prob;
    StepControl *ctl;
    const long long *x0, *y0;  // [np + 1] item prefix counts of the sweeps
    const int *rb0, *ib0;      // [np + 1] block prefix counts of the ghost and init kernels
    int np;
    long long x_total, y_total;
    int ring_blocks, init_blocks;
    int grid_x, grid_y;        // sweep grids (blocks); 0 = all resident blocks
};

#define FVM2D_DECLARE_BATCH_VARIANT(ns)                                        \
    namespace ns {                                                             \
    cudaError_t batch_prepare(int *occ_x, int *occ_y);                         \
    cudaError_t batch_enqueue_init(const BatchLaunch &L, cudaStream_t s);      \
    cudaError_t batch_enqueue_plan(const BatchLaunch &L, cudaStream_t s);      \
    cudaError_t batch_enqueue_step(const BatchLaunch &L, cudaStream_t s);      \
    }

FVM2D_DECLARE_BATCH_VARIANT(fp64)
FVM2D_DECLARE_BATCH_VARIANT(fp64_strict)
FVM2D_DECLARE_BATCH_VARIANT(fp64_reforder)
FVM2D_DECLARE_BATCH_VARIANT(fp32)

} // namespace fvm2d
