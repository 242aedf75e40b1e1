// fvm2d_adjoint.cu -- the adjoint step in FP64 (namespace adj).
#define FVM2D_VARIANT adj
#define FVM2D_REAL double
#include "fvm2d_adjoint.inc"
#include "fvm2d_adjoint_launch.inc"
