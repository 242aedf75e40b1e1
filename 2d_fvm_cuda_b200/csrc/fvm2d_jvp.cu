// fvm2d_jvp.cu -- tangent-linear build: the FP64 kernels with shared
// reciprocals (Hoisted) instantiated on dual numbers, so every state value
// carries a tangent through the same arithmetic (forward-mode
// differentiation of the step, almost everywhere).
#include "fvm2d_dual.cuh"
#define FVM2D_VARIANT jvp
#define FVM2D_REAL fvm2d::ad::Dual
#define FVM2D_PHYS Hoisted
#define FVM2D_X_MINB 2
#define FVM2D_Y_MINB 2
#include "fvm2d_variant.inc"
