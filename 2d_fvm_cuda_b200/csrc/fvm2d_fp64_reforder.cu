// fvm2d_fp64_reforder.cu -- FP64 kernels in the reference's operation order
// with nvcc's default FMA contraction (FVM2D_FP64_REFORDER): the arithmetic
// the reference's own build performs, up to the compiler's contraction
// choices.
#define FVM2D_VARIANT fp64_reforder
#define FVM2D_REAL double
#define FVM2D_PHYS RefOrder
// resident sweep blocks per SM (128 threads each) that the register
// budget is fitted to; measured best for this build at 4096^2
#define FVM2D_X_MINB 4
#define FVM2D_Y_MINB 4
#include "fvm2d_variant.inc"
