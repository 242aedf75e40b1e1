// fvm2d_fp64_strict.cu -- FP64 kernels compiled with -fmad=false: every
// operation rounds separately, in the reference's order, so results agree bit
// for bit with the reference built with -fmad=false and with the CPU oracle.
#define FVM2D_VARIANT fp64_strict
#define FVM2D_REAL double
#include "fvm2d_variant.inc"
