// fvm2d_fp64.cu -- FP64 kernels with hoisted reciprocals and FMA contraction:
// the product default (FVM2D_FP64).  Checked against the reference within a
// relative L1 tolerance.
#define FVM2D_VARIANT fp64
#define FVM2D_REAL double
#define FVM2D_PHYS Hoisted
#define FVM2D_TAPED_STEP  // also the taped step of the differentiation form
// reciprocals and reciprocal square roots from the hardware seeds and one
// third-order refinement (rrcp/rrsqrt in fvm2d_math.cuh)
#define FVM2D_FAST_RCP
// resident sweep blocks per SM (128 threads each) that the register
// budget is fitted to; measured best for this build at 4096^2
#ifdef FVM2D_TUNE_X
#define FVM2D_X_MINB FVM2D_TUNE_X
#define FVM2D_Y_MINB FVM2D_TUNE_Y
#else
#define FVM2D_X_MINB 5
#define FVM2D_Y_MINB 5
#endif
#include "fvm2d_variant.inc"
