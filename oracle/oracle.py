"""ctypes access to the checker libraries (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this
module.  The product (the `2d_fvm_cuda_b200` package and libfvm2d.so) never
does.

* ``Oracle``  -- oracle/_build/liboracle.so, the C restatement of the
  reference's step (src/basicFuns.cuh, src/ghostCellPresets.cuh,
  src/wrappers.cuh:196-284).
* ``RefHost`` -- oracle/_ref/libref_host.so, the reference's own kernels
  compiled for the host and driven in the launch order of
  src/wrappers.cuh:154-306 (present only where the reference sources were
  available at build time).
* ``run_ref_gpu`` -- oracle/_ref/ref_gpu[_nofma], the reference's own CUDA
  kernels on the GPU (needs a GPU).

States are numpy arrays of shape (ny, nx, 4) float64 holding (rho, p, u, v).
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_HOST_SO = os.path.join(HERE, "_ref", "libref_host.so")
REF_GPU = os.path.join(HERE, "_ref", "ref_gpu")
REF_GPU_NOFMA = os.path.join(HERE, "_ref", "ref_gpu_nofma")

# ghostCellStrategy codes (src/wrappers.cuh:17-24) plus the two new presets.
OUTFLOW, REFLECTIVE, JET, JET800, DOUBLE_MACH, PERIODIC, REFLECTIVE_TB = range(7)

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class _Params(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("width", ctypes.c_double), ("height", ctypes.c_double),
        ("cfl", ctypes.c_double), ("alpha", ctypes.c_double),
        ("gamma", ctypes.c_double), ("t_end", ctypes.c_double),
        ("strategy", ctypes.c_int),
    ]


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _state(U) -> np.ndarray:
    U = np.ascontiguousarray(U, dtype=np.float64).copy()
    if U.ndim != 3 or U.shape[2] != 4:
        raise ValueError("state must have shape (ny, nx, 4)")
    return U


def build_oracle() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


class Oracle:
    """The C restatement.  Methods return new arrays; inputs are not modified."""

    def __init__(self, threads: int = 0):
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        lib = ctypes.CDLL(ORACLE_SO)
        lib.orc_max_speed.restype = ctypes.c_double
        lib.orc_max_speed.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double]
        lib.orc_step.restype = ctypes.c_int
        lib.orc_step.argtypes = [_dp, ctypes.POINTER(_Params), _dp, _dp]
        lib.orc_solve.restype = ctypes.c_int
        lib.orc_solve.argtypes = [_dp, ctypes.POINTER(_Params), ctypes.c_int, _ip, _dp]
        lib.orc_ghost.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                  ctypes.c_double, ctypes.c_double, ctypes.c_int]
        for name in ("orc_sweep_x", "orc_sweep_y"):
            getattr(lib, name).argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double]
        lib.orc_slope.argtypes = [_dp, _dp, _dp, ctypes.c_double, ctypes.c_double, _dp]
        lib.orc_grp.argtypes = [_dp, _dp, _dp, _dp, ctypes.c_double, _dp, _dp]
        lib.orc_flux.argtypes = [_dp, _dp, ctypes.c_double, _dp]
        lib.orc_set_threads.argtypes = [ctypes.c_int]
        lib.orc_set_threads(threads)
        self.lib = lib

    @staticmethod
    def params(nx, ny, width=1.0, height=1.0, cfl=0.5, alpha=1.9, gamma=1.4,
               t_end=0.0, strategy=OUTFLOW) -> _Params:
        return _Params(nx, ny, width, height, cfl, alpha, gamma, t_end, strategy)

    def max_speed(self, U, gamma=1.4) -> float:
        U = _state(U)
        return self.lib.orc_max_speed(_ptr(U), U.shape[1], U.shape[0], gamma)

    def sweep_x(self, U, width, dt, alpha=1.9, gamma=1.4):
        U = _state(U)
        self.lib.orc_sweep_x(_ptr(U), U.shape[1], U.shape[0], width, dt, alpha, gamma)
        return U

    def sweep_y(self, U, height, dt, alpha=1.9, gamma=1.4):
        U = _state(U)
        self.lib.orc_sweep_y(_ptr(U), U.shape[1], U.shape[0], height, dt, alpha, gamma)
        return U

    def ghost(self, U, strategy, t=0.0, width=1.0, height=1.0):
        U = _state(U)
        self.lib.orc_ghost(_ptr(U), U.shape[1], U.shape[0], width, height, t, strategy)
        return U

    def step(self, U, t=0.0, **kw):
        """One step from time t.  Returns (U_new, t_new, dt) or None when the loop has ended."""
        U = _state(U)
        p = self.params(U.shape[1], U.shape[0], **kw)
        tt = ctypes.c_double(t)
        dt = ctypes.c_double(0.0)
        if self.lib.orc_step(_ptr(U), ctypes.byref(p), ctypes.byref(tt), ctypes.byref(dt)):
            return None
        return U, tt.value, dt.value

    def solve(self, U, max_steps=-1, **kw):
        """Runs from t=0 until the loop ends.  Returns (U, steps, t)."""
        U = _state(U)
        p = self.params(U.shape[1], U.shape[0], **kw)
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        self.lib.orc_solve(_ptr(U), ctypes.byref(p), max_steps, ctypes.byref(steps), ctypes.byref(t))
        return U, steps.value, t.value


class RefHost:
    """The reference's own kernels on the host (oracle/_ref/libref_host.so)."""

    def __init__(self, threads: int = 0):
        if not os.path.exists(REF_HOST_SO):
            raise FileNotFoundError(REF_HOST_SO)
        lib = ctypes.CDLL(REF_HOST_SO)
        lib.ref_run.restype = ctypes.c_int
        lib.ref_run.argtypes = [_dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_int, ctypes.c_double, ctypes.c_int, _ip, _dp]
        lib.ref_set_threads.argtypes = [ctypes.c_int]
        lib.ref_set_threads(threads)
        self.lib = lib

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_HOST_SO)

    def run(self, U, width=1.0, height=1.0, cfl=0.5, alpha=1.9, gamma=1.4, t_end=0.0,
            strategy=OUTFLOW, t0=0.0, max_steps=-1):
        """Returns (U, steps, t)."""
        U = _state(U)
        steps = ctypes.c_int(0)
        t = ctypes.c_double(0.0)
        rc = self.lib.ref_run(_ptr(U), U.shape[1], U.shape[0], width, height, cfl, alpha, gamma,
                              t_end, strategy, t0, max_steps, ctypes.byref(steps), ctypes.byref(t))
        if rc:
            raise ValueError("reference host run rejected the case (sizes must be multiples of 16)")
        return U, steps.value, t.value


def run_ref_gpu(U, width=1.0, height=1.0, cfl=0.5, alpha=1.9, gamma=1.4, t_end=0.0,
                strategy=OUTFLOW, max_steps=-1, fma=True):
    """Runs the reference's CUDA kernels (needs a GPU).

    Returns (U, steps, t, loop_ms, kernel_ms) where loop_ms is the reference's
    own std::chrono timer around its loop (wrappers.cuh:193,286-288)."""
    exe = REF_GPU if fma else REF_GPU_NOFMA
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    U = _state(U)
    ny, nx, _ = U.shape
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        with open(fin, "wb") as f:
            f.write(struct.pack("4i", nx, ny, strategy, max_steps))
            f.write(struct.pack("6d", width, height, cfl, alpha, gamma, t_end))
            f.write(U.tobytes())
        subprocess.run([exe, fin, fout], check=True)
        with open(fout, "rb") as f:
            steps, _pad = struct.unpack("2i", f.read(8))
            t, loop_ms, kernel_ms = struct.unpack("3d", f.read(24))
            out = np.frombuffer(f.read(), dtype=np.float64).reshape(ny, nx, 4).copy()
    return out, steps, t, loop_ms, kernel_ms
