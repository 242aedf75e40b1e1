"""The per-cell device code of the step that runs without exchanges between
threads -- the ghost-ring rules (ghost_cell), the step-size plan
(plan_step) and the wave speed -- compiled for the host from
2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh (tests/kernels_host.cpp) and
compared with the oracle bit for bit, without a GPU:

* the ghost fill on all seven presets, odd and even sizes, several times
  (the double-Mach shock moves with t), and the ring's wave-speed maximum;
* the same fill in the row frames of slabs (global row numbers for the jet
  rows and the shock, only the problem's own edges filled);
* the step size and end-of-loop decision of the reference's rule
  (src/wrappers.cuh:196-207, the oracle's orc_dt).
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


@pytest.fixture(scope="module")
def kh(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    so = str(tmp_path_factory.mktemp("kernels_host") / "libkernels_host.so")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I", CUDA_INC,
                    os.path.join(HERE, "kernels_host.cpp"), "-o", so], check=True)
    lib = ctypes.CDLL(so)
    lib.kh_ghost.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.c_void_p]
    lib.kh_plan.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p]
    lib.kh_wave_speed.argtypes = [ctypes.c_long, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    return lib


def ghost(kh, U, strategy, t, row0=0, gny=None, top=True, bottom=True, gamma=1.4):
    V = np.ascontiguousarray(U[..., :4], dtype=np.float64).copy()
    ny, nx = V.shape[:2]
    vmax = ctypes.c_double(0.0)
    assert kh.kh_ghost(V.ctypes.data, nx, ny, strategy, gamma, t, row0, gny or ny, int(top), int(bottom),
                       ctypes.byref(vmax)) == 0
    return V, vmax.value


def ring_mask(ny, nx):
    m = np.zeros((ny, nx), bool)
    m[:2] = m[-2:] = True
    m[:, :2] = m[:, -2:] = True
    return m


@pytest.mark.parametrize("strategy", range(7))
def test_ghost_fill_equals_the_oracle(kh, oracle, pkg, strategy):
    for nx, ny in [(48, 32), (37, 29), (64, 64), (100, 36), (6, 6)]:
        U = pkg.scenarios.seeded_four_quadrant(nx, ny, 11 + nx)
        for t in (0.0, 0.013, 0.1):
            G, vmax = ghost(kh, U, strategy, t)
            R = oracle.ghost(U, strategy, t=t)
            assert np.array_equal(G, R, equal_nan=True), (nx, ny, t)
            ring = np.ascontiguousarray(R[ring_mask(ny, nx)][None])
            assert vmax == oracle.max_speed(ring), (nx, ny, t)


@pytest.mark.parametrize("strategy", range(7))
def test_ghost_fill_in_slab_row_frames(kh, oracle, pkg, strategy):
    """Each rank's fill of its rows equals the whole problem's fill there:
    ring columns on the rows it owns, ring rows only on the problem's own
    edges; halo rows are left as they were."""
    sl = pkg.slab
    for nx, ny, world in [(48, 40, 2), (40, 50, 3), (36, 44, 4)]:
        U = pkg.scenarios.seeded_four_quadrant(nx, ny, 5 * world + strategy)
        t = 0.02
        R = oracle.ghost(U, strategy, t=t)
        for rank in range(world):
            l_lo, l_hi = sl.local_rows(ny, world, rank)
            row0, gny, top, bottom = sl.row_frame(ny, world, rank, strategy)
            S = U[l_lo:l_hi]
            G, _ = ghost(kh, S, strategy, t, row0, gny, top, bottom)
            a = 0 if top else 2
            b = len(S) - (0 if bottom else 2)
            assert np.array_equal(G[a:b], R[l_lo + a:l_lo + b], equal_nan=True), (world, rank)
            assert np.array_equal(G[:a], S[:a, :, :4]) and np.array_equal(G[b:], S[b:, :, :4]), (world, rank)


def test_step_size_plan_equals_the_reference_rule(kh, oracle, pkg):
    """plan_step from the committed state's wave-speed max against the
    oracle's orc_dt on the same state: dt bit for bit, and the same end of
    the loop (t past the end time, or h / smax below 1e-20)."""
    lib = oracle.lib
    lib.orc_dt.restype = ctypes.c_int
    lib.orc_dt.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    rng = np.random.default_rng(4)
    for k in range(400):
        nx, ny = int(rng.integers(6, 40)), int(rng.integers(6, 40))
        U = np.ascontiguousarray(pkg.scenarios.seeded_four_quadrant(nx, ny, k)[..., :4])
        if k % 50 == 0:
            U[..., 2] *= 1e25  # wave speeds past the 1e-20 break
        width, height = rng.uniform(0.1, 3.0, 2)
        cfl, t_end = rng.uniform(0.05, 0.9), rng.uniform(0.0, 0.5)
        t = [0.0, t_end, rng.uniform(0, t_end), t_end - 1e-12, t_end + 1e-3][k % 5]
        p = oracle.params(nx, ny, width=width, height=height, cfl=cfl, t_end=t_end)
        odt = ctypes.c_double(-1.0)
        ended = lib.orc_dt(U.ctypes.data, ctypes.byref(p), t, ctypes.byref(odt))
        smax = oracle.max_speed(U)
        hmin = min(width / nx, height / ny)
        dt, active, done = ctypes.c_double(0), ctypes.c_int(0), ctypes.c_int(0)
        kh.kh_plan(t, smax, 0, 1 << 30, 0, t_end, cfl, hmin, 0.0, ctypes.byref(dt), ctypes.byref(active),
                   ctypes.byref(done))
        assert bool(done.value) == bool(ended) and bool(active.value) == (not ended), k
        if not ended:
            assert dt.value == odt.value, k


def test_step_plan_limits_and_fixed_step(kh):
    dt, active, done = ctypes.c_double(0), ctypes.c_int(0), ctypes.c_int(0)
    args = (ctypes.byref(dt), ctypes.byref(active), ctypes.byref(done))
    kh.kh_plan(0.1, 2.0, 7, 7, 0, 1.0, 0.5, 0.01, 0.0, *args)  # step limit reached: idle, not ended
    assert (active.value, done.value) == (0, 0)
    kh.kh_plan(0.1, 2.0, 3, 7, 1, 1.0, 0.5, 0.01, 0.0, *args)  # ended stays ended
    assert (active.value, done.value) == (0, 1)
    kh.kh_plan(5.0, 2.0, 3, 7, 0, 1.0, 0.5, 0.01, 1e-3, *args)  # fixed dt: the end time does not apply
    assert (active.value, done.value, dt.value) == (1, 0, 1e-3)


def test_wave_speed_equals_the_oracle(kh, oracle, pkg):
    U = np.ascontiguousarray(pkg.scenarios.seeded_four_quadrant(300, 200, 9)[..., :4])
    out = np.empty(300 * 200)
    kh.kh_wave_speed(out.size, U.ctypes.data, 1.4, out.ctypes.data)
    assert out.max() == oracle.max_speed(U)
    for row in (0, 57, 199):
        assert out.reshape(200, 300)[row].max() == oracle.max_speed(np.ascontiguousarray(U[row:row + 1]))
