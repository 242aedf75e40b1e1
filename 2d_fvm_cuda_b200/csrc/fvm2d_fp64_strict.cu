// fvm2d_fp64_strict.cu -- FP64 kernels in the reference's operation order,
// compiled with -fmad=false (FVM2D_FP64_STRICT): every operation rounds on its
// own, in the reference's order, so results agree bit for bit with the
// reference built with -fmad=false and with the CPU oracle.
#define FVM2D_VARIANT fp64_strict
#define FVM2D_REAL double
#define FVM2D_PHYS RefOrder
// resident sweep blocks per SM (128 threads each) that the register
// budget is fitted to; measured best for this build at 4096^2
#define FVM2D_X_MINB 4
#define FVM2D_Y_MINB 4
#include "fvm2d_variant.inc"
