"""Python mirror of the reference's solver class over the C ABI.

`RGRP_2D_CUDA` keeps the names, argument meaning and call order of the
reference's C++ class (src/wrappers.cuh:26-65) so code written against it
reads the same; the work happens in libfvm2d.so on the GPU.
"""
from __future__ import annotations

import enum
import os

import numpy as np

from . import _lib


class ghostCellStrategy(enum.IntEnum):
    """src/wrappers.cuh:17-24, plus two presets the reference does not have."""
    outflow = 0
    reflective = 1     # the reference runs its double-Mach preset for it (wrappers.cuh:277-280)
    jet = 2
    jet800 = 3
    doubleMach = 4
    periodic = 5       # two-layer wrap in both directions
    reflective_tb = 6  # reflecting top/bottom walls, transmissive left/right


class precision(enum.IntEnum):
    fp64 = _lib.FP64                    # shared reciprocals + FMA: fastest, within relative L1 1e-10
    fp64_strict = _lib.FP64_STRICT      # reference order, no contraction: bit-exact with the reference -fmad=false
    fp64_reforder = _lib.FP64_REFORDER  # reference order with FMA contraction, as the reference's own build
    fp32 = _lib.FP32                    # FP32 storage/arithmetic, compensated update, FP64 dt
    fp32_residual = _lib.FP32_RESIDUAL  # FP32 arithmetic, FP32 + 16-bit residual planes, FP64 update


def write_matrix_txt(dir: str, U, t: float) -> None:
    """src/wrappers.cuh:370-397 (writeMatrixTo_txt): rho_/p_/u_/v_<t>s.txt in
    `dir`, the time formatted as std::to_string(double) does ("%f"), one text
    row per grid row of U (ny, nx, 4|5), each value in the default stream
    format (6 significant digits, "%g") followed by a space."""
    tag = "%f" % t
    names = ("rho", "p", "u", "v")
    files = [open(os.path.join(dir, f"{n}_{tag}s.txt"), "w") for n in names]
    try:
        for row in U:
            for k, f in enumerate(files):
                f.write("".join("%g " % x for x in row[:, k]))
                f.write("\n")
    finally:
        for f in files:
            f.close()


class RGRP_2D_CUDA:
    """Split 2D Euler solver: MUSCL + generalized minmod + relaxation GRP.

    States are arrays of shape (Ny, Nx, 4) = (rho, p, u, v) or (Ny, Nx, 5)
    (the reference's vec5d rows), ghost layers included.
    """

    def __init__(self, U0=None):
        # defaults of src/wrappers.cuh:49-52
        self._width, self._height = 1.0, 1.0
        self._end_time, self._cfl = 0.0, 0.5
        self._alpha, self._gamma = 1.9, 1.4
        self._nx, self._ny = 100, 100
        self._strategy = ghostCellStrategy.outflow
        self._precision = precision.fp64
        self._U0 = None
        self._U = None
        self._ms = 0.0
        self._stages = 0
        self._handle = None
        if U0 is not None:
            A = np.asarray(U0, dtype=np.float64)
            if A.ndim != 3 or A.shape[2] not in (4, 5):
                raise ValueError("U0 must be (Ny, Nx, 4) or (Ny, Nx, 5)")
            self._U0 = np.ascontiguousarray(A[:, :, :4])
            self._ny, self._nx = A.shape[0], A.shape[1]

    # -- setters: src/wrappers.cuh:80-152 --------------------------------
    def setRPInitialData(self, U1, U2, U3, U4, Nx: int, Ny: int) -> None:
        """Four constant states: U2 | U1 over U3 | U4 (src/wrappers.cuh:80-108)."""
        U = np.empty((Ny, Nx, 4))
        hx, hy = Nx // 2, Ny // 2
        U[:hy, :hx] = np.asarray(U2, dtype=np.float64)[:4]
        U[hy:, :hx] = np.asarray(U3, dtype=np.float64)[:4]
        U[:hy, hx:] = np.asarray(U1, dtype=np.float64)[:4]
        U[hy:, hx:] = np.asarray(U4, dtype=np.float64)[:4]
        self._U0, self._nx, self._ny = U, Nx, Ny

    def setSpatialLayout(self, width: float, height: float) -> None:
        self._width, self._height = float(width), float(height)

    def setTimeLayout(self, endTime: float, CFL: float | None = None) -> None:
        self._end_time = float(endTime)
        if CFL is not None:
            self._cfl = float(CFL)

    def setCFL(self, CFL: float) -> None:
        self._cfl = float(CFL)

    def setAlpha(self, alpha: float) -> None:
        self._alpha = float(alpha)

    def setGamma(self, gamma: float) -> None:
        self._gamma = float(gamma)

    def setGhostCellStrategy(self, strategy) -> None:
        self._strategy = ghostCellStrategy(strategy)

    def setPrecision(self, p) -> None:
        """Arithmetic build (no reference counterpart)."""
        self._precision = precision(p)

    def setRecordModel(self, on_off: bool, gapPerFrame: int = 10, recordDir: str = ".") -> None:
        """PNG frames during solve() (src/wrappers.cuh:147-152): <recordDir>/<k>.png
        after step k for k = 0, gapPerFrame, 2 gapPerFrame, ..., density in
        viridis over its range (rendered on the GPU, written without OpenCV)."""
        self._record = (bool(on_off), int(gapPerFrame), str(recordDir))

    # -- solve: src/wrappers.cuh:154-306 ----------------------------------
    def _get_handle(self) -> _lib.Handle:
        h = self._handle
        if h is None or (h.nx, h.ny) != (self._nx, self._ny):
            if h is not None:
                h.close()
            h = self._handle = _lib.Handle(self._nx, self._ny)
        h.configure(self._width, self._height, self._end_time, self._cfl, self._alpha, self._gamma,
                    int(self._strategy), int(self._precision))
        h.set_record_model(*getattr(self, "_record", (False, 10, ".")))
        return h

    def solve(self) -> np.ndarray:
        """Runs from t = 0 to the end time; returns the (Ny, Nx, 5) vec5d rows.

        Like the reference (src/wrappers.cuh:290), the result also becomes
        the initial data of a later solve()."""
        if self._U0 is None:
            raise RuntimeError("no initial data: pass U0 or call setRPInitialData first")
        h = self._get_handle()
        h.set_state(self._U0)
        h.solve()
        self._ms = h.computation_time_ms()
        self._stages += h.time()[1]
        U = h.get_state(5)
        self._U0 = np.ascontiguousarray(U[:, :, :4])
        self._U = U
        return U

    def getComputationTime_ms(self) -> float:
        return self._ms

    def getTimeStagesCount(self) -> int:
        return self._stages

    def getConservedTotals(self) -> np.ndarray:
        """Mass, x momentum, y momentum and energy of the last result's
        interior cells, summed in FP64 (fvm2d_get_conserved_totals; no
        reference counterpart)."""
        if self._handle is None or self._U is None:
            raise RuntimeError("no result: call solve() first")
        return self._handle.conserved_totals()

    def writeFinalResultTo_txt(self, dir: str) -> None:
        """rho_/p_/u_/v_<endTime>s.txt of the last result
        (src/wrappers.cuh:318-321); see write_matrix_txt."""
        if self._U is None:
            return
        write_matrix_txt(dir, self._U, self._end_time)

    def clear(self) -> None:
        """src/wrappers.cuh:347-353."""
        self._U0 = None
        self._U = None
        if self._handle is not None:
            self._handle.close()
            self._handle = None
