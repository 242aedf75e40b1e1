"""B200-native split 2D Euler finite-volume solver (sm_100a kernels behind a C ABI).

The package directory name starts with a digit, so import it with
``importlib.import_module("2d_fvm_cuda_b200")``.

* ``RGRP_2D_CUDA``, ``ghostCellStrategy``, ``precision`` -- the reference's
  solver interface (src/wrappers.cuh:17-65) over libfvm2d.so.
* ``Handle`` -- one C-ABI solver handle (include/fvm2d.h), for callers that
  want the state to stay on the GPU between calls.
* ``Batch`` -- many independent problems of different sizes solved together.
* ``slab`` -- one problem split by rows across processes (one GPU each).
* ``ensemble`` -- many independent problems dealt out whole across processes
  (one GPU each), each rank's share solved as one batch.
* ``scenarios`` -- initial data (the reference's demo problems and seeded
  workloads).
"""
from . import ensemble, scenarios, slab  # noqa: F401
from ._lib import (FP32, FP32_RESIDUAL, FP64, FP64_REFORDER, FP64_STRICT, FULL_TAPE, LIB_PATH, Batch,  # noqa: F401
                   FVM2DError, Handle, load, measure_fp64_peak)
from .solver import RGRP_2D_CUDA, ghostCellStrategy, precision  # noqa: F401
