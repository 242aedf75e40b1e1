// fvm2d_control.h -- records shared by every build of the kernels and the host runtime.
#pragma once

#include <cuda_runtime.h>

namespace fvm2d {

// Device-resident loop state, one per solver handle.  The kernels of a step
// read the step size from it and the step's last kernel advances it, so the
// time loop of src/wrappers.cuh:196-284 runs without a host round trip.
struct StepControl {
    double t;                      // committed simulation time
    double dt;                     // step size of the step in flight
    double smax_last;              // max wave speed of the committed state
    unsigned long long smax_bits;  // running max (bit pattern of a non-negative double)
    int steps;                     // committed steps
    int step_limit;                // no step starts once `steps` reaches this
    int active;                    // 1 while a step is in flight
    int done;                      // 1 once the loop of wrappers.cuh:196 has ended
    unsigned int ticket;           // last-block detection in grid reductions
    int first_bad;                 // 1-based step that first left an interior cell with NaN or
                                   // non-positive density or pressure; 0: none
};

struct PlanParams {
    double t_end;     // end time
    double cfl;       // CFL number
    double hmin;      // min(width/nx, height/ny), wrappers.cuh:202
    double fixed_dt;  // > 0: every step uses this dt (no CFL rule), for differentiation
};

// Everything one build of the kernels needs to enqueue a step.
struct LaunchConfig {
    int nx, ny, pitch;
    long long plane;       // elements between field planes
    void *U, *A, *B;       // state buffers: U holds the state, A and B are sweep scratch
    StepControl *ctl;
    double hx, hy;         // width/nx, height/ny
    double rhx, rhy;       // 1.0/hx, 1.0/hy
    double alpha, gamma;
    int strategy;
    PlanParams plan;
    // Row frame when the array is one row slab of a larger one (a problem
    // split across processes): the global row of local row 0, the global row
    // count (0: ny), and whether the preset fills the top ghost rows (0, 1)
    // and the bottom ones.  Ring rows it does not fill are halo rows, left out
    // of the wave-speed max.
    int row0 = 0, ny_global = 0, fill_top = 1, fill_bottom = 1;
};

// Kernels per step: sweep X, sweep Y, sweep Y, sweep X + average, ghost ring.
constexpr int kStepKernels = 5;

// x-sweep work items: a warp walks `chunks` chunks of 32 cells of one row and
// updates 32 chunks - 2 cells (the first chunk's first two lanes only feed
// their neighbours).  Item seg of a row updates cells 2 + cells seg ..
// 1 + cells (seg + 1).  Long items waste less; an array must still give
// every resident warp a couple of items, so the chunk count is the largest
// of 8, 4, 2, 1 that does (x_chunks_for).
__host__ __device__ constexpr int x_item_cells(int chunks) { return 32 * chunks - 2; }
__host__ __device__ constexpr int x_items_per_row(int nx, int chunks)
{
    return (nx - 4 + x_item_cells(chunks) - 1) / x_item_cells(chunks);
}
inline int x_chunks_for(long long rows, int nx, long long resident_warps)
{
    int c = 8;
    while (c > 1 && rows * x_items_per_row(nx, c) < 2 * resident_warps) c /= 2;
    return c;
}

// The entry points each build of the kernels provides (namespaces fp64,
// fp64_strict, fp64_reforder, fp32, and jvp: FP64 values with tangents).
#define FVM2D_DECLARE_VARIANT(ns)                                              \
    namespace ns {                                                             \
    cudaError_t prepare();                                                     \
    cudaError_t enqueue_init(const LaunchConfig &c, cudaStream_t s);           \
    cudaError_t enqueue_plan(const LaunchConfig &c, cudaStream_t s);           \
    cudaError_t enqueue_plan_from(const LaunchConfig &c, cudaStream_t s, const double *smax); \
    cudaError_t enqueue_step(const LaunchConfig &c, cudaStream_t s, cudaEvent_t *ev); \
    }

FVM2D_DECLARE_VARIANT(fp64)
FVM2D_DECLARE_VARIANT(fp64_strict)
FVM2D_DECLARE_VARIANT(fp64_reforder)
FVM2D_DECLARE_VARIANT(fp32)
FVM2D_DECLARE_VARIANT(fp32r)
FVM2D_DECLARE_VARIANT(jvp)

// The FP64 and FP32 steps keeping what their adjoint needs: X(U) in c.A, Y(U)
// in c.B and the interface fluxes of the four sweeps (X of U, Y of U, Y of A,
// X of B), each stored at the interface's right cell in planes mass, normal
// momentum, energy, tangential momentum.  The step reads c.U and writes its
// result to `out` (c.U when null).
namespace fp64 {
cudaError_t enqueue_step_taped(const LaunchConfig &c, cudaStream_t s, void *const flux[4], void *out);
}
namespace fp32 {
cudaError_t enqueue_step_taped(const LaunchConfig &c, cudaStream_t s, void *const flux[4], void *out);
}

// Records `msg` as the calling thread's fvm2d_last_error() text; returns code.
int report_error(int code, const char *msg);

} // namespace fvm2d
