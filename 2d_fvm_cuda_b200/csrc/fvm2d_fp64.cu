// fvm2d_fp64.cu -- FP64 kernels, nvcc default FMA contraction (the product
// build; the reference's own build contracts the same way by default).
#define FVM2D_VARIANT fp64
#define FVM2D_REAL double
#include "fvm2d_variant.inc"
