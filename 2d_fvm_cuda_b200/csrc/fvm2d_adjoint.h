// fvm2d_adjoint.h -- entry points of the adjoint step (fvm2d_adjoint.inc,
// built as fvm2d_adjoint.cu in FP64 and fvm2d_adjoint32.cu in FP32).
#pragma once

#include <cuda_runtime.h>

namespace fvm2d {

// One reverse step of a build with shared reciprocals at fixed dt, from the
// tape of its forward step (enqueue_step_taped of fp64 or fp32).  All buffers
// are state-sized, 4 planes of pitch x ny values of the build's type.
struct AdjointLaunch {
    int nx, ny, pitch, strategy;
    long long plane;
    double hx, hy, rhx, rhy, alpha, gamma, dt;
    const void *U;         // input state of the step
    const void *A1, *B1;   // X(U) and Y(U)
    const void *flux[4];   // interface fluxes of the sweeps X(U), Y(U), Y(A1), X(B1)
    const void *lb_out;    // adjoint of the step's output state
    void *lb_in;           // result: adjoint of the input state (may not alias lb_out)
    void *work[4];         // work states (the fourth used with a fork stream)
    // optional: a second stream and two events of the caller's; branch B's
    // first sweep transpose then runs on `fork` beside branch A's two, so
    // the transposes fill each other's tail waves (also inside a graph
    // capture, as parallel branches)
    cudaStream_t fork = nullptr;
    cudaEvent_t fork_ev[2] = {nullptr, nullptr};
};

#define FVM2D_DECLARE_ADJOINT(ns)                                                 \
    namespace ns {                                                                \
    /* Queries the device once (SM count, occupancy); call before capturing    \
       adjoint steps into a graph.  adjoint_step calls it too. */               \
    cudaError_t adjoint_prepare();                                                \
    cudaError_t adjoint_step(const AdjointLaunch &L, cudaStream_t s);            \
    }

FVM2D_DECLARE_ADJOINT(adj)    // FP64
FVM2D_DECLARE_ADJOINT(adj32)  // FP32

} // namespace fvm2d
