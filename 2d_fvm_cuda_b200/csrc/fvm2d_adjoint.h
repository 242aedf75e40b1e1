// fvm2d_adjoint.h -- entry point of the adjoint step (fvm2d_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

namespace fvm2d {

// One reverse step of the FP64 build with shared reciprocals at fixed dt, from
// the tape of its forward step (fp64::enqueue_step_taped).  All buffers are
// state-sized: 4 planes of pitch x ny doubles.
struct AdjointLaunch {
    int nx, ny, pitch, strategy;
    long long plane;
    double hx, hy, rhx, rhy, alpha, gamma, dt;
    const double *U;        // input state of the step
    const double *A1, *B1;  // X(U) and Y(U)
    const double *flux[4];  // interface fluxes of the sweeps X(U), Y(U), Y(A1), X(B1)
    const double *lb_out;   // adjoint of the step's output state
    double *lb_in;          // result: adjoint of the input state (may not alias lb_out)
    double *work[3];        // work states
};

// Queries the device once (SM count, occupancy); call before capturing
// adjoint steps into a graph.  adjoint_step calls it too.
cudaError_t adjoint_prepare();

cudaError_t adjoint_step(const AdjointLaunch &L, cudaStream_t s);

} // namespace fvm2d
