// fvm2d_adjoint32.cu -- the adjoint step in FP32 (namespace adj32), for the
// FP32 build's differentiation runs.  Built like fvm2d_fp32.cu with
// single-precision division and square root within 2 ulp.
#define FVM2D_VARIANT adj32
#define FVM2D_REAL float
#include "fvm2d_adjoint.inc"
#include "fvm2d_adjoint_launch.inc"
