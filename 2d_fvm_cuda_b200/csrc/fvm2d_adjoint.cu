// fvm2d_adjoint.cu -- the adjoint step in FP64 (namespace adj).
#define FVM2D_VARIANT adj
#define FVM2D_REAL double
// the forward recomputed with the FP64 product build's reciprocals
#define FVM2D_FAST_RCP
#include "fvm2d_adjoint.inc"
#include "fvm2d_adjoint_launch.inc"
