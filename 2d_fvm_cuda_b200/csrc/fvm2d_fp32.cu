// fvm2d_fp32.cu -- FP32 storage and arithmetic (FVM2D_FP32): the hoisted
// physics in single precision with the compensated conservative update, the
// update and face states in packed FP32x2 instructions; the
// wave-speed reduction, dt and time stay in FP64.  Reports its error against
// the FP64 path rather than matching the reference bit for bit.  Built with
// -prec-div=false -prec-sqrt=false (FP32 division and square root within
// 2 ulp).
#define FVM2D_VARIANT fp32
#define FVM2D_REAL float
#define FVM2D_PHYS PackedCompensated
#define FVM2D_TAPED_STEP  // also the taped step of FP32 differentiation runs
// the FP64 wave speed from reciprocal square roots (fvm2d_math.cuh)
#define FVM2D_FAST_RCP
// resident sweep blocks per SM (128 threads each) that the register
// budget is fitted to
#ifdef FVM2D_TUNE_X
#define FVM2D_X_MINB FVM2D_TUNE_X
#define FVM2D_Y_MINB FVM2D_TUNE_Y
#else
#define FVM2D_X_MINB 6
#define FVM2D_Y_MINB 6
#endif
#include "fvm2d_packed.cuh"
#include "fvm2d_variant.inc"
