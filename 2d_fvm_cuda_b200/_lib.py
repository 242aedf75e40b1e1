"""ctypes binding of lib/libfvm2d.so (the C ABI declared in include/fvm2d.h).

The library is built in-tree (`make -C 2d_fvm_cuda_b200`).  There is no
fallback: if the shared object is missing or a call fails, an exception
says why.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "lib", "libfvm2d.so")

FVM2D_OK, FVM2D_ERR_INVALID, FVM2D_ERR_CUDA, FVM2D_ERR_STATE = 0, 1, 2, 3
FP64, FP64_STRICT, FP64_REFORDER, FP32, FP32_RESIDUAL = 0, 1, 2, 3, 4
FULL_TAPE = 0  # fvm2d_forward(checkpoints=FULL_TAPE): tape every step, no recompute in vjp

_dp = ctypes.POINTER(ctypes.c_double)
_vp = ctypes.c_void_p

# (name, restype, argtypes) of every entry point in include/fvm2d.h
SIGNATURES = [
    ("fvm2d_last_error", ctypes.c_char_p, []),
    ("fvm2d_version", ctypes.c_char_p, []),
    ("fvm2d_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int]),
    ("fvm2d_destroy", ctypes.c_int, [_vp]),
    ("fvm2d_set_spatial_layout", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    ("fvm2d_set_time_layout", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double]),
    ("fvm2d_set_end_time", ctypes.c_int, [_vp, ctypes.c_double]),
    ("fvm2d_set_cfl", ctypes.c_int, [_vp, ctypes.c_double]),
    ("fvm2d_set_alpha", ctypes.c_int, [_vp, ctypes.c_double]),
    ("fvm2d_set_gamma", ctypes.c_int, [_vp, ctypes.c_double]),
    ("fvm2d_set_ghost_strategy", ctypes.c_int, [_vp, ctypes.c_int]),
    ("fvm2d_set_precision", ctypes.c_int, [_vp, ctypes.c_int]),
    ("fvm2d_set_state", ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    ("fvm2d_set_state_planes", ctypes.c_int, [_vp, _vp]),
    ("fvm2d_get_state_planes", ctypes.c_int, [_vp, _vp]),
    ("fvm2d_set_rp_initial_data", ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    ("fvm2d_get_state", ctypes.c_int, [_vp, _vp, ctypes.c_int]),
    ("fvm2d_solve", ctypes.c_int, [_vp]),
    ("fvm2d_advance", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_get_health", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_get_conserved_totals", ctypes.c_int, [_vp, _dp]),
    ("fvm2d_set_record_model", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]),
    ("fvm2d_write_frame_png", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("fvm2d_write_state", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("fvm2d_read_state", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("fvm2d_advance_dt", ctypes.c_int, [_vp, ctypes.c_double]),
    ("fvm2d_get_wave_speed_max", ctypes.c_int, [_vp, _dp]),
    ("fvm2d_set_row_frame", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("fvm2d_get_rows", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    ("fvm2d_set_rows", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    ("fvm2d_get_stream", ctypes.c_int, [_vp, ctypes.POINTER(_vp)]),
    ("fvm2d_get_rows_async", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    ("fvm2d_set_rows_async", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp]),
    ("fvm2d_slab_begin", ctypes.c_int, [_vp, _vp]),
    ("fvm2d_slab_step", ctypes.c_int, [_vp, _vp, _vp]),
    ("fvm2d_slab_sync", ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_get_computation_time_ms", ctypes.c_int, [_vp, _dp]),
    ("fvm2d_get_time_stages_count", ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_longlong)]),
    ("fvm2d_get_time", ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_int), _dp]),
    ("fvm2d_get_run_stats", ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_longlong)]),
    ("fvm2d_profile_kernels", ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_measure_fp64_peak", ctypes.c_int, [_dp, _dp]),
    ("fvm2d_eval_reciprocals", ctypes.c_int, [_vp, ctypes.c_longlong, _vp, _vp]),
    ("fvm2d_set_fixed_dt", ctypes.c_int, [_vp, ctypes.c_double]),
    ("fvm2d_set_vjp_overlap", ctypes.c_int, [_vp, ctypes.c_int]),
    ("fvm2d_jvp", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int]),
    ("fvm2d_forward", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    ("fvm2d_vjp", ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int]),
    ("fvm2d_batch_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_batch_destroy", ctypes.c_int, [_vp]),
    ("fvm2d_batch_set_problem", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                               ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]),
    ("fvm2d_batch_set_precision", ctypes.c_int, [_vp, ctypes.c_int]),
    ("fvm2d_batch_set_state", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    ("fvm2d_batch_get_state", ctypes.c_int, [_vp, ctypes.c_int, _vp, ctypes.c_int]),
    ("fvm2d_batch_solve", ctypes.c_int, [_vp]),
    ("fvm2d_batch_get_time", ctypes.c_int, [_vp, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_batch_get_run_stats", ctypes.c_int, [_vp, _dp, ctypes.POINTER(ctypes.c_longlong),
                                                 ctypes.POINTER(ctypes.c_longlong)]),
    ("fvm2d_batch_autotune", ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                            ctypes.POINTER(ctypes.c_int)]),
    ("fvm2d_advance_noalloc", ctypes.c_int,
     [_vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
      ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_int, _vp, _dp,
      ctypes.POINTER(ctypes.c_int)]),
]

_LIB = None


class FVM2DError(RuntimeError):
    """A libfvm2d call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libfvm2d error {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    """Loads libfvm2d.so once; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                "(the CUDA library is required; there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = lib
    return _LIB


def check(rc: int) -> None:
    if rc != FVM2D_OK:
        raise FVM2DError(rc, load().fvm2d_last_error().decode())


def measure_fp64_peak() -> tuple[float, float]:
    """(TFLOP/s, ms per launch) of fvm2d_measure_fp64_peak on the current device."""
    lib = load()
    tf, ms = ctypes.c_double(0), ctypes.c_double(0)
    check(lib.fvm2d_measure_fp64_peak(ctypes.byref(tf), ctypes.byref(ms)))
    return tf.value, ms.value


def as_cells(U) -> np.ndarray:
    """(ny, nx, 4|5) float64 C-contiguous view/copy of a state."""
    A = np.ascontiguousarray(U, dtype=np.float64)
    if A.ndim != 3 or A.shape[2] not in (4, 5):
        raise ValueError("a state is an array of shape (ny, nx, 4) or (ny, nx, 5)")
    return A


class Handle:
    """Owns one fvm2d_solver.  Thin: every method is one C call."""

    def __init__(self, nx: int, ny: int):
        self.lib = load()
        self.nx, self.ny = int(nx), int(ny)
        h = _vp()
        check(self.lib.fvm2d_create(ctypes.byref(h), self.nx, self.ny))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.fvm2d_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def configure(self, width=1.0, height=1.0, t_end=0.0, cfl=0.5, alpha=1.9, gamma=1.4,
                  strategy=0, precision=FP64) -> None:
        check(self.lib.fvm2d_set_spatial_layout(self.h, width, height))
        check(self.lib.fvm2d_set_time_layout(self.h, t_end, cfl))
        check(self.lib.fvm2d_set_alpha(self.h, alpha))
        check(self.lib.fvm2d_set_gamma(self.h, gamma))
        check(self.lib.fvm2d_set_ghost_strategy(self.h, int(strategy)))
        check(self.lib.fvm2d_set_precision(self.h, int(precision)))

    def set_state(self, U) -> None:
        A = as_cells(U)
        if A.shape[:2] != (self.ny, self.nx):
            raise ValueError(f"state shape {A.shape[:2]} does not match ({self.ny}, {self.nx})")
        check(self.lib.fvm2d_set_state(self.h, A.ctypes.data, A.shape[2]))

    def set_state_ptr(self, ptr: int, stride: int) -> None:
        """Uploads from a raw host or device pointer of ny*nx*stride doubles."""
        check(self.lib.fvm2d_set_state(self.h, ptr, stride))

    def get_state(self, stride: int = 4, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((self.ny, self.nx, stride))
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.shape == (self.ny, self.nx, stride)
        check(self.lib.fvm2d_get_state(self.h, out.ctypes.data, stride))
        return out

    def set_state_planes(self, planes) -> None:
        """Uploads a (4, ny, nx) array of planes rho, p, u, v."""
        P = np.ascontiguousarray(planes, dtype=np.float64)
        assert P.shape == (4, self.ny, self.nx)
        check(self.lib.fvm2d_set_state_planes(self.h, P.ctypes.data))

    def get_state_planes(self) -> np.ndarray:
        out = np.empty((4, self.ny, self.nx))
        check(self.lib.fvm2d_get_state_planes(self.h, out.ctypes.data))
        return out

    def set_state_planes_ptr(self, ptr: int) -> None:
        """From host or device memory at ptr: 4*ny*nx doubles, planes rho, p, u, v."""
        check(self.lib.fvm2d_set_state_planes(self.h, ptr))

    def get_state_planes_ptr(self, ptr: int) -> None:
        check(self.lib.fvm2d_get_state_planes(self.h, ptr))

    def get_state_ptr(self, ptr: int, stride: int) -> None:
        check(self.lib.fvm2d_get_state(self.h, ptr, stride))

    def solve(self) -> None:
        check(self.lib.fvm2d_solve(self.h))

    def advance(self, n: int) -> int:
        k = ctypes.c_int(0)
        check(self.lib.fvm2d_advance(self.h, int(n), ctypes.byref(k)))
        return k.value

    def time(self):
        t = ctypes.c_double(0)
        s = ctypes.c_int(0)
        dt = ctypes.c_double(0)
        check(self.lib.fvm2d_get_time(self.h, ctypes.byref(t), ctypes.byref(s), ctypes.byref(dt)))
        return t.value, s.value, dt.value

    def computation_time_ms(self) -> float:
        ms = ctypes.c_double(0)
        check(self.lib.fvm2d_get_computation_time_ms(self.h, ctypes.byref(ms)))
        return ms.value

    def run_stats(self):
        """(device_ms, kernel_launches) of the last solve()/advance() loop."""
        ms = ctypes.c_double(0)
        n = ctypes.c_longlong(0)
        check(self.lib.fvm2d_get_run_stats(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def profile_kernels(self, nsteps: int):
        """Mean per-kernel times (ms) over up to nsteps steps: [sweep X, sweep Y,
        sweep Y, sweep X + average, ghost ring], and the steps taken."""
        out = (ctypes.c_double * 5)()
        k = ctypes.c_int(0)
        check(self.lib.fvm2d_profile_kernels(self.h, int(nsteps), out, ctypes.byref(k)))
        return list(out), k.value

    def first_bad_step(self) -> int:
        """1-based step that first left a NaN or non-positive density or
        pressure in an interior cell since the state was set; 0: none."""
        k = ctypes.c_int(0)
        check(self.lib.fvm2d_get_health(self.h, ctypes.byref(k)))
        return k.value

    def conserved_totals(self) -> np.ndarray:
        """Mass, x momentum, y momentum and energy of the interior cells, in
        FP64 whatever the precision (fvm2d_get_conserved_totals)."""
        out = np.zeros(4)
        check(self.lib.fvm2d_get_conserved_totals(self.h, out.ctypes.data_as(_dp)))
        return out

    # -- frames and state files --
    def set_record_model(self, on: bool, gap_per_frame: int = 10, record_dir: str = ".") -> None:
        """Frames <record_dir>/<k>.png during solve(), every gap_per_frame steps."""
        check(self.lib.fvm2d_set_record_model(self.h, int(bool(on)), int(gap_per_frame),
                                              os.fsencode(record_dir)))

    def write_frame_png(self, path: str) -> None:
        check(self.lib.fvm2d_write_frame_png(self.h, os.fsencode(path)))

    def write_state(self, path: str) -> None:
        check(self.lib.fvm2d_write_state(self.h, os.fsencode(path)))

    def read_state(self, path: str) -> None:
        check(self.lib.fvm2d_read_state(self.h, os.fsencode(path)))

    # -- row slabs (one problem split across processes) --
    def advance_dt(self, dt: float) -> None:
        """One step with the caller's dt."""
        check(self.lib.fvm2d_advance_dt(self.h, float(dt)))

    def wave_speed_max(self) -> float:
        v = ctypes.c_double(0)
        check(self.lib.fvm2d_get_wave_speed_max(self.h, ctypes.byref(v)))
        return v.value

    def set_row_frame(self, row0: int, ny_global: int, fill_top: bool, fill_bottom: bool) -> None:
        check(self.lib.fvm2d_set_row_frame(self.h, int(row0), int(ny_global), int(bool(fill_top)),
                                           int(bool(fill_bottom))))

    def get_rows(self, j0: int, nrows: int, out: np.ndarray | None = None) -> np.ndarray:
        """Rows j0 .. j0+nrows-1 as a (4, nrows, nx) array (planes rho, p, u, v)."""
        if out is None:
            out = np.empty((4, nrows, self.nx))
        assert out.dtype == np.float64 and out.flags["C_CONTIGUOUS"] and out.size == 4 * nrows * self.nx
        check(self.lib.fvm2d_get_rows(self.h, int(j0), int(nrows), out.ctypes.data))
        return out

    def set_rows(self, j0: int, rows: np.ndarray) -> None:
        R = np.ascontiguousarray(rows, dtype=np.float64)
        nrows = R.size // (4 * self.nx)
        assert R.size == 4 * nrows * self.nx
        check(self.lib.fvm2d_set_rows(self.h, int(j0), int(nrows), R.ctypes.data))

    def get_rows_ptr(self, j0: int, nrows: int, ptr: int) -> None:
        """As get_rows, into host or device memory at ptr (4*nrows*nx doubles)."""
        check(self.lib.fvm2d_get_rows(self.h, int(j0), int(nrows), ptr))

    def set_rows_ptr(self, j0: int, nrows: int, ptr: int) -> None:
        check(self.lib.fvm2d_set_rows(self.h, int(j0), int(nrows), ptr))

    # asynchronous slab steps: enqueued on the handle's stream, no host wait
    def stream_ptr(self) -> int:
        """The handle's cudaStream_t (for torch.cuda.ExternalStream)."""
        p = ctypes.c_void_p(0)
        check(self.lib.fvm2d_get_stream(self.h, ctypes.byref(p)))
        return p.value or 0

    def get_rows_async(self, j0: int, nrows: int, ptr: int) -> None:
        check(self.lib.fvm2d_get_rows_async(self.h, int(j0), int(nrows), ptr))

    def set_rows_async(self, j0: int, nrows: int, ptr: int) -> None:
        check(self.lib.fvm2d_set_rows_async(self.h, int(j0), int(nrows), ptr))

    def slab_begin(self, smax_out_ptr: int) -> None:
        check(self.lib.fvm2d_slab_begin(self.h, smax_out_ptr))

    def slab_step(self, smax_in_ptr: int, smax_out_ptr: int) -> None:
        check(self.lib.fvm2d_slab_step(self.h, smax_in_ptr, smax_out_ptr))

    def slab_sync(self):
        """(t, steps, done) after the enqueued slab steps have run."""
        t, k, d = ctypes.c_double(0), ctypes.c_int(0), ctypes.c_int(0)
        check(self.lib.fvm2d_slab_sync(self.h, ctypes.byref(t), ctypes.byref(k), ctypes.byref(d)))
        return t.value, k.value, bool(d.value)

    # -- differentiation (fixed dt; forward/vjp on FP64 or FP32, jvp on FP64) --
    def set_fixed_dt(self, dt: float) -> None:
        check(self.lib.fvm2d_set_fixed_dt(self.h, float(dt)))

    def set_vjp_overlap(self, on: bool) -> None:
        """Two tape buffers in vjp(), the next segment recomputed while the
        current one is reversed (the default), or one buffer taking turns."""
        check(self.lib.fvm2d_set_vjp_overlap(self.h, int(bool(on))))

    def jvp(self, nsteps: int, tangent) -> np.ndarray:
        """Advances nsteps carrying `tangent`; returns the final tangent."""
        T = as_cells(tangent)
        out = np.empty((self.ny, self.nx, T.shape[2]))
        check(self.lib.fvm2d_jvp(self.h, int(nsteps), T.ctypes.data, out.ctypes.data, T.shape[2]))
        return out

    def forward(self, nsteps: int, checkpoints: int) -> None:
        """nsteps steps keeping `checkpoints` states for vjp(), or with
        checkpoints=FULL_TAPE the whole tape (7 states per step)."""
        check(self.lib.fvm2d_forward(self.h, int(nsteps), int(checkpoints)))

    def vjp(self, cotangent) -> np.ndarray:
        """Cotangent of the initial state of the last forward() for `cotangent` of its final state."""
        C = as_cells(cotangent)
        out = np.empty((self.ny, self.nx, C.shape[2]))
        check(self.lib.fvm2d_vjp(self.h, C.ctypes.data, out.ctypes.data, C.shape[2]))
        return out

    def time_stages_count(self) -> int:
        c = ctypes.c_longlong(0)
        check(self.lib.fvm2d_get_time_stages_count(self.h, ctypes.byref(c)))
        return c.value


class Batch:
    """Owns one fvm2d_batch: many problems of different sizes solved together."""

    def __init__(self, sizes):
        """sizes: sequence of (nx, ny)."""
        self.lib = load()
        self.sizes = [(int(a), int(b)) for a, b in sizes]
        n = len(self.sizes)
        nx = (ctypes.c_int * n)(*[s[0] for s in self.sizes])
        ny = (ctypes.c_int * n)(*[s[1] for s in self.sizes])
        h = _vp()
        check(self.lib.fvm2d_batch_create(ctypes.byref(h), n, nx, ny))
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.fvm2d_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_problem(self, p, width=1.0, height=1.0, t_end=0.0, cfl=0.5, alpha=1.9, gamma=1.4, strategy=0):
        check(self.lib.fvm2d_batch_set_problem(self.h, p, width, height, t_end, cfl, alpha, gamma, int(strategy)))

    def set_precision(self, precision: int) -> None:
        check(self.lib.fvm2d_batch_set_precision(self.h, int(precision)))

    def set_state(self, p, U) -> None:
        A = as_cells(U)
        if A.shape[:2] != (self.sizes[p][1], self.sizes[p][0]):
            raise ValueError("state shape does not match the problem size")
        check(self.lib.fvm2d_batch_set_state(self.h, p, A.ctypes.data, A.shape[2]))

    def get_state(self, p, stride: int = 4) -> np.ndarray:
        nx, ny = self.sizes[p]
        out = np.empty((ny, nx, stride))
        check(self.lib.fvm2d_batch_get_state(self.h, p, out.ctypes.data, stride))
        return out

    def solve(self) -> None:
        check(self.lib.fvm2d_batch_solve(self.h))

    def time(self, p):
        t = ctypes.c_double(0)
        k = ctypes.c_int(0)
        check(self.lib.fvm2d_batch_get_time(self.h, p, ctypes.byref(t), ctypes.byref(k)))
        return t.value, k.value

    def run_stats(self):
        """(device_ms, kernel_launches, cell_updates) of the last solve."""
        ms = ctypes.c_double(0)
        n = ctypes.c_longlong(0)
        c = ctypes.c_longlong(0)
        check(self.lib.fvm2d_batch_get_run_stats(self.h, ctypes.byref(ms), ctypes.byref(n), ctypes.byref(c)))
        return ms.value, n.value, c.value

    def autotune(self, trial_steps: int = 2):
        """Picks the y-segment length and sweep grid size; returns them."""
        T = ctypes.c_int(0)
        g = ctypes.c_int(0)
        check(self.lib.fvm2d_batch_autotune(self.h, int(trial_steps), ctypes.byref(T), ctypes.byref(g)))
        return T.value, g.value
