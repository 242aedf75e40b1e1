// fvm2d_fp32r.cu -- FP32 arithmetic on FP32 states with 16-bit residual
// planes (FVM2D_FP32_RESIDUAL): slopes, the relaxation GRP and the fluxes in
// single precision from the FP32 plane values, and the conservative update
// of each cell in FP64 from its stored hi + lo, split back into the FP32 and
// residual planes (fvm2d_split.cuh).  The rounding of the stored state --
// which, not the FP32 arithmetic, dominates the FP32 build's distance from
// FP64 over long runs -- drops from 2^-24 to about 2^-32 relative.  Built
// with -prec-div=false -prec-sqrt=false, as FVM2D_FP32.
#define FVM2D_VARIANT fp32r
#define FVM2D_REAL float
#define FVM2D_PHYS PackedResidual
#define FVM2D_NO_BATCH  // the batched form runs FP64 and FP32 only
// the FP64 wave speed and the update's reciprocal from the refined hardware
// seeds (fvm2d_math.cuh)
#define FVM2D_FAST_RCP
#ifdef FVM2D_TUNE_X
#define FVM2D_X_MINB FVM2D_TUNE_X
#define FVM2D_Y_MINB FVM2D_TUNE_Y
#else
#define FVM2D_X_MINB 6
#define FVM2D_Y_MINB 6
#endif
#include "fvm2d_packed.cuh"
#include "fvm2d_variant.inc"
