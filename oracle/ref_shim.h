/*
 * ref_shim.h -- lets a host C++ compiler build the reference's device code
 * (src/basicFuns.cuh, src/ghostCellPresets.cuh) unchanged, so the checker can
 * run the reference's own per-cell routines on CPU cores.
 *
 * TEST INFRASTRUCTURE ONLY.  Force-included (-include) ahead of the
 * reference headers by oracle/Makefile; nothing in the product uses it.
 * cuda_runtime.h under a non-CUDA compiler defines __global__/__device__ as
 * empty; the launch indices become thread-local globals that the emulated
 * launches in ref_host.cpp set before every call; thrust::swap on doubles and
 * the unqualified sqrt/abs calls resolve to the host versions.
 */
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <thrust/swap.h>
extern thread_local uint3 threadIdx, blockIdx;
extern thread_local dim3 blockDim;
using std::sqrt;
using std::abs;
