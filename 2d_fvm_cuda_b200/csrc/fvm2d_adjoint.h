// fvm2d_adjoint.h -- entry point of the adjoint step (fvm2d_adjoint.cu).
#pragma once

#include <cuda_runtime.h>

namespace fvm2d {

// One reverse step of the FP64 build with shared reciprocals at fixed dt.
// All buffers are state-sized: 4 planes of pitch x ny doubles.
struct AdjointLaunch {
    int nx, ny, pitch, strategy;
    long long plane;
    double hx, hy, rhx, rhy, alpha, gamma, dt;
    double *U;         // input state of the step
    double *lb_out;    // adjoint of the step's output state
    double *lb_in;     // result: adjoint of the input state (may not alias lb_out)
    double *state[6];  // work: A1, B1, the transposed ghost/average, three sweep adjoints
    double *work[7];   // work of a sweep transpose: fluxes, cell parts, update adjoints, 4 interface adjoints
};

cudaError_t adjoint_step(const AdjointLaunch &L, cudaStream_t s);

} // namespace fvm2d
