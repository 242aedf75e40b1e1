"""The device code of the step's kernels -- the sweep work items (x_item
with its lanes' shuffles run by a 32-thread host warp, y_item), the
ghost-ring rules (ghost_cell), the step-size plan (plan_step) and the wave
speed -- compiled for the host from 2d_fvm_cuda_b200/csrc/fvm2d_kernels.cuh
(tests/kernels_host.cpp) and compared with the oracle bit for bit, without a
GPU:

* x and y sweeps through the kernels' own work items and item numbering
  (30-cell row segments; 32-column segments of T interfaces for every T the
  kernels choose), the final x-sweep averaging in place, and a whole step
  composed as the kernels run it, in the reference's operation order
  (RefOrder, what the contraction-free build runs); the shared-reciprocal
  items within rounding, and the FP32 build's items (PackedCompensated,
  32-bit plane offsets) within single-precision rounding;

* the ghost fill on all seven presets, odd and even sizes, several times
  (the double-Mach shock moves with t), and the ring's wave-speed maximum;
* the same fill in the row frames of slabs (global row numbers for the jet
  rows and the shock, only the problem's own edges filled);
* the step size and end-of-loop decision of the reference's rule
  (src/wrappers.cuh:196-207, the oracle's orc_dt);
* whole solves through the single-problem kernels (sweep_x_kernel,
  sweep_y_kernel, ghost_kernel with its last-block step commit, init_kernel)
  on every preset, and their health record of the first bad step;
* frames: the density range and viridis kernels and the PNG writer
  (2d_fvm_cuda_b200/csrc/fvm2d_io.cuh) against a numpy rendering, the file
  decoded with zlib (CRCs, Adler-32, stored blocks above 64 KiB);
* the batched kernels (2d_fvm_cuda_b200/csrc/fvm2d_batch.cuh: problem
  lookup, item chunks per warp across problem boundaries, per-problem step
  control, tickets and wave-speed maxima, skipped items of finished
  problems) solving six problems of mixed sizes and presets, each equal to
  the oracle's solve of that problem alone;
* the adjoint step's own kernels (2d_fvm_cuda_b200/csrc/fvm2d_adjoint.inc:
  the x and y sweep transposes, with the y tiles in shared memory and block
  barriers, and the ghost-ring transposes) as the transpose of the
  dual-number tangent of the forward work items, on every preset:
  <J v, w> = <v, J^T w>; and the FP32 build's adjoint (the same kernels in
  single precision after its taped FP32 forward, tests/adjoint32_host.cpp)
  against the FP64 one.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")


def build_host(tmp_path_factory, source, defines=()):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    so = str(tmp_path_factory.mktemp("kernels_host") / (os.path.splitext(source)[0] + ".so"))
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-pthread",
                    *[f"-D{d}" for d in defines], "-I", CUDA_INC, os.path.join(HERE, source), "-o", so],
                   check=True)
    return ctypes.CDLL(so)


STEP_ARGS = [ctypes.c_void_p] * 2 + [ctypes.c_int] * 3 + [ctypes.c_double] * 6 + [ctypes.c_int]


@pytest.fixture(scope="module")
def k32(tmp_path_factory):
    lib = build_host(tmp_path_factory, "adjoint32_host.cpp")
    lib.k32_step_vjp.argtypes = STEP_ARGS + [ctypes.c_void_p]
    return lib


def _kernels_host(tmp_path_factory, defines=()):
    lib = build_host(tmp_path_factory, "kernels_host.cpp", defines)
    lib.kh_ghost.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                             ctypes.c_void_p]
    lib.kh_plan.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                            ctypes.c_void_p, ctypes.c_void_p]
    lib.kh_wave_speed.argtypes = [ctypes.c_long, ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]
    lib.kh_sweep.argtypes = [ctypes.c_int] * 4 + [ctypes.c_void_p] * 3 + [ctypes.c_int] * 2 + [ctypes.c_double] * 4
    lib.kh_solve.argtypes = ([ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 +
                             [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4)
    lib.kh_solve_build.argtypes = ([ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 6 +
                                   [ctypes.c_int] * 4 + [ctypes.c_void_p] * 4)
    lib.kh_frame.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    lib.kh_batch_solve.argtypes = ([ctypes.c_int] + [ctypes.c_void_p] * 4 + [ctypes.c_int] * 4 +
                                   [ctypes.c_void_p] * 3)
    lib.kh_sweep32.argtypes = [ctypes.c_int] * 3 + [ctypes.c_void_p] * 3 + [ctypes.c_int] * 2 + [ctypes.c_double] * 4
    lib.kh_step_jvp.argtypes = STEP_ARGS + [ctypes.c_void_p] * 2
    lib.kh_step_vjp.argtypes = STEP_ARGS + [ctypes.c_void_p]
    lib.kh_totals.argtypes = ([ctypes.c_void_p] + [ctypes.c_int] * 5 + [ctypes.c_double] * 2 + [ctypes.c_void_p])
    return lib


@pytest.fixture(scope="module")
def kh(tmp_path_factory):
    return _kernels_host(tmp_path_factory)


@pytest.fixture(scope="module")
def kh_fast(tmp_path_factory):
    """The same device code with FVM2D_FAST_RCP, as the FP64 product build is
    compiled: reciprocals and reciprocal square roots from a seed refined by
    one third-order step (on the host the seed is a single-precision one)."""
    return _kernels_host(tmp_path_factory, ("FVM2D_FAST_RCP",))


REF, HOISTED, REF_RING, REF_XRING = 0, 1, 2, 3
ALPHA, GAMMA = 1.9, 1.4


def sweep(kh, policy, direction, U, h, dt, T=16, comb=None):
    """direction 0: x-sweep items, 1: y-sweep items of T interfaces; comb:
    the final x-sweep, averaging with comb in place."""
    U = np.ascontiguousarray(U[..., :4], dtype=np.float64)
    ny, nx = U.shape[:2]
    out = np.empty_like(U)
    cb = None if comb is None else np.ascontiguousarray(comb[..., :4], dtype=np.float64)
    assert kh.kh_sweep(policy, direction, int(comb is not None), T, U.ctypes.data,
                       None if cb is None else cb.ctypes.data, out.ctypes.data, nx, ny, h, dt, ALPHA, GAMMA) == 0
    return out


SWEEP_SIZES = [(48, 32), (37, 29), (33, 7), (6, 6), (70, 12), (300, 9)]


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


def sweep_case(pkg, oracle, nx, ny, seed):
    U = oracle.ghost(pkg.scenarios.seeded_four_quadrant(nx, ny, seed), 0)
    width, height = 1.0, 1.1
    dt = 0.3 * min(width / nx, height / ny) / oracle.max_speed(U)
    return U, width, height, dt


@pytest.mark.parametrize("nx,ny", SWEEP_SIZES)
def test_sweep_items_equal_the_oracle_sweeps(kh, oracle, pkg, nx, ny):
    U, width, height, dt = sweep_case(pkg, oracle, nx, ny, 3)
    X = sweep(kh, REF, 0, U, width / nx, dt)
    assert np.array_equal(X, oracle.sweep_x(U, width, dt))  # every cell written, bit for bit
    # the x walker that streams its row through the shared-memory ring
    assert np.array_equal(sweep(kh, REF_XRING, 0, U, width / nx, dt), X)
    # x items of every length the kernels choose (chunks of 32 cells per item)
    for chunks in (1, 4, 8):
        assert kh.kh_set_xchunks(chunks) == 0
        try:
            assert np.array_equal(sweep(kh, REF, 0, U, width / nx, dt), X), chunks
            assert np.array_equal(sweep(kh, REF_XRING, 0, U, width / nx, dt), X), chunks
        finally:
            kh.kh_set_xchunks(2)
    RY = oracle.sweep_y(U, height, dt)
    for T in (8, 16, 32, 64, 4):  # the kernels choose 64, 32, 16 or 8; 4 for short segments
        assert np.array_equal(sweep(kh, REF, 1, U, height / ny, dt, T), RY), T
        # the walker that streams its columns through the shared-memory ring
        assert np.array_equal(sweep(kh, REF_RING, 1, U, height / ny, dt, T), RY), T


@pytest.mark.parametrize("fast", [False, True], ids=["ieee_division", "refined_reciprocals"])
@pytest.mark.parametrize("nx,ny", SWEEP_SIZES[:3])
def test_hoisted_sweep_items_agree_to_rounding(kh, kh_fast, oracle, pkg, nx, ny, fast):
    U, width, height, dt = sweep_case(pkg, oracle, nx, ny, 4)
    cases = ((0, oracle.sweep_x(U, width, dt), width / nx), (1, oracle.sweep_y(U, height, dt), height / ny))
    for direction, R, h in cases:
        H = sweep(kh_fast if fast else kh, HOISTED, direction, U, h, dt)
        rel = np.abs(H - R).max(axis=(0, 1)) / np.abs(R).max(axis=(0, 1))
        assert rel.max() <= 1e-13, (direction, rel)  # measured 1.5e-16 (IEEE division)


def normwise(A, R):
    return (np.abs(A - R) / (np.abs(R) + np.median(np.abs(R), axis=(0, 1)))).max()


@pytest.mark.parametrize("nx,ny", SWEEP_SIZES[:4])
def test_fp32_sweep_items_stay_within_single_precision(kh, oracle, pkg, nx, ny):
    """The FP32 build's items on FP32 values against the oracle's FP64 sweeps
    of the same values: about one FP32 rounding (measured 8.7e-8)."""
    U, width, height, dt = sweep_case(pkg, oracle, nx, ny, 5)
    U = np.ascontiguousarray(U.astype(np.float32).astype(np.float64))

    def sweep32(direction, V, h, T=16, comb=None):
        out = np.empty_like(V)
        cb = None if comb is None else np.ascontiguousarray(comb)
        assert kh.kh_sweep32(direction, int(comb is not None), T, V.ctypes.data,
                             None if cb is None else cb.ctypes.data, out.ctypes.data, nx, ny, h, dt, ALPHA,
                             GAMMA) == 0
        return out

    assert normwise(sweep32(0, U, width / nx), oracle.sweep_x(U, width, dt)) <= 5e-7
    RY = oracle.sweep_y(U, height, dt)
    for T in (8, 16, 32, 64):
        assert normwise(sweep32(1, U, height / ny, T), RY) <= 5e-7, T
    A = np.ascontiguousarray(RY.astype(np.float32).astype(np.float64))
    F = sweep32(0, U, width / nx, comb=A)
    assert normwise(F, (oracle.sweep_x(U, width, dt) + A) * 0.5) <= 5e-7


@pytest.mark.parametrize("strategy", [0, 4, 5])
def test_one_step_composed_from_the_kernels_items(kh, oracle, pkg, strategy):
    """The step as the kernels run it: X(U) -> A, Y(U) -> B, Y(A) -> U, the
    final sweep X(B) averaged with U in place, then the ghost fill at the
    advanced time; against the oracle's step."""
    nx, ny = 45, 31
    U = oracle.ghost(pkg.scenarios.seeded_four_quadrant(nx, ny, 12 + strategy), strategy)
    kw = dict(width=1.0, height=0.8, cfl=0.45, alpha=ALPHA, gamma=GAMMA, t_end=1.0, strategy=strategy)
    for _ in range(3):
        R, t1, dt = oracle.step(U, t=0.0, **kw)
        A = sweep(kh, REF, 0, U, kw["width"] / nx, dt)
        B = sweep(kh, REF, 1, U, kw["height"] / ny, dt, T=8)
        V = sweep(kh, REF, 1, A, kw["height"] / ny, dt, T=8)
        V = sweep(kh, REF, 0, B, kw["width"] / nx, dt, comb=V)
        V, _ = ghost(kh, V, strategy, t1)
        assert np.array_equal(V, R)
        U = R


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


def adjoint_case(oracle, pkg, strategy, nx=37, ny=29, width=1.0, height=0.8):
    """A four-quadrant state with every cell perturbed (no cell pair exactly
    equal, so no limiter or wave-case test sits on its switch)."""
    rng = np.random.default_rng(strategy)
    U = oracle.ghost(pkg.scenarios.seeded_four_quadrant(nx, ny, 40 + strategy), strategy)
    noise = rng.standard_normal((2,) + U.shape) * 0.05
    U = np.ascontiguousarray(U * (1 + noise[0] * [1, 1, 0, 0]) + noise[1] * [0, 0, 1, 1])
    dt = 0.3 * min(width / nx, height / ny) / oracle.max_speed(U)
    return U, dt, rng


@pytest.mark.parametrize("strategy,nx,ny", [(s, 37, 29) for s in range(7)] + [(0, 300, 263), (5, 259, 301)])
def test_adjoint_kernels_transpose_the_forward_items(kh, oracle, pkg, strategy, nx, ny):
    """One step: the tangent J v from the forward items on dual numbers and
    the cotangent J^T w from the adjoint kernels satisfy <J v, w> =
    <v, J^T w> to rounding; the dual run's values are the step itself
    (checked against the oracle).  The larger arrays take many work items
    per line."""
    width, height, t = 1.0, 0.8, 0.01
    U, dt, rng = adjoint_case(oracle, pkg, strategy, nx, ny)
    v = np.ascontiguousarray(rng.standard_normal(U.shape))
    w = np.ascontiguousarray(rng.standard_normal(U.shape))
    out, Jv, JTw = np.empty_like(U), np.empty_like(U), np.empty_like(U)
    args = (nx, ny, strategy, t, dt, width, height, ALPHA, GAMMA, 8)
    assert kh.kh_step_jvp(U.ctypes.data, v.ctypes.data, *args, out.ctypes.data, Jv.ctypes.data) == 0
    assert kh.kh_step_vjp(U.ctypes.data, w.ctypes.data, *args, JTw.ctypes.data) == 0
    # the value part: the shared-reciprocal step, against the oracle's sweeps and fill
    A = oracle.sweep_y(oracle.sweep_x(U, width, dt), height, dt)
    B = oracle.sweep_x(oracle.sweep_y(U, height, dt), width, dt)
    R = oracle.ghost((A + B) * 0.5, strategy, t=t + dt, width=width, height=height)
    assert np.abs(out - R).max() <= 1e-12 * np.abs(R).max()
    a, b = np.sum(Jv * w), np.sum(v * JTw)
    assert abs(a - b) <= 1e-13 * max(abs(a), abs(b)), (a, b)  # measured <= 1.6e-15


@pytest.mark.parametrize("grid", [(1, 1), (3, 2)], ids=["one-block", "several-blocks"])
def test_batched_kernels_equal_single_solves(kh, oracle, grid):
    """Six problems of different sizes, presets and end times (the first one
    ends after two steps, so its items are skipped afterwards) through the
    batched kernels, 12 steps; each problem against the oracle alone."""
    import ensemble_ranks

    probs = ensemble_ranks.problems()[:6]
    steps = 12
    keys = ("width", "height", "t_end", "cfl", "alpha", "gamma", "strategy")
    nx = np.array([U.shape[1] for U, _ in probs], dtype=np.int32)
    ny = np.array([U.shape[0] for U, _ in probs], dtype=np.int32)
    par = np.array([[kw[k] for k in keys] for _, kw in probs], dtype=np.float64)
    cells = np.concatenate([np.ascontiguousarray(U[..., :4]).ravel() for U, _ in probs])
    out, t, n = np.empty_like(cells), np.empty(len(probs)), np.empty(len(probs), dtype=np.int32)
    assert kh.kh_batch_solve(len(probs), nx.ctypes.data, ny.ctypes.data, par.ctypes.data, cells.ctypes.data, 16,
                             grid[0], grid[1], steps, out.ctypes.data, t.ctypes.data, n.ctypes.data) == 0
    c = 0
    for p, (U, kw) in enumerate(probs):
        size = 4 * U.shape[0] * U.shape[1]
        G = out[c:c + size].reshape(U.shape[0], U.shape[1], 4)
        c += size
        R, rsteps, rt = oracle.solve(U, max_steps=steps, **kw)
        assert (int(n[p]), float(t[p])) == (rsteps, rt), p
        assert np.array_equal(G, R, equal_nan=True), p
    assert n[0] < steps  # one problem finished early and was skipped


def kernel_solve(kh, U, kw, blocks, max_steps, T=16):
    U = np.ascontiguousarray(U[..., :4], dtype=np.float64)
    ny, nx = U.shape[:2]
    out = np.empty_like(U)
    t, steps, bad = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    assert kh.kh_solve(U.ctypes.data, nx, ny, kw["width"], kw["height"], kw["t_end"], kw["cfl"], kw["alpha"],
                       kw["gamma"], kw["strategy"], T, blocks, max_steps, out.ctypes.data, ctypes.byref(t),
                       ctypes.byref(steps), ctypes.byref(bad)) == 0
    return out, steps.value, t.value, bad.value


def build_solve(kh, build, U, kw, blocks, max_steps, T=16):
    """kh_solve through a build's physics: 0 FP64 (Hoisted), 1 FP32, 2 FP32
    with residual planes."""
    U = np.ascontiguousarray(U[..., :4], dtype=np.float64)
    ny, nx = U.shape[:2]
    out = np.empty_like(U)
    t, steps, bad = ctypes.c_double(), ctypes.c_int(), ctypes.c_int()
    assert kh.kh_solve_build(build, U.ctypes.data, nx, ny, kw["width"], kw["height"], kw["t_end"], kw["cfl"],
                             kw["alpha"], kw["gamma"], kw["strategy"], T, blocks, max_steps, out.ctypes.data,
                             ctypes.byref(t), ctypes.byref(steps), ctypes.byref(bad)) == 0
    return out, steps.value, t.value, bad.value


@pytest.mark.parametrize("strategy", range(7))
def test_single_problem_kernels_solve_like_the_oracle(kh, oracle, pkg, strategy):
    """init_kernel, then the five kernels of a step as the step graphs launch
    them, until the device control record ends the loop (the end time, for
    the presets whose loops end before 15 steps) or 15 steps; one and three
    blocks per sweep."""
    nx, ny = 41, 30
    U = pkg.scenarios.seeded_four_quadrant(nx, ny, 60 + strategy)
    if strategy in (5, 6):
        U = oracle.ghost(U, strategy)
    kw = dict(width=1.0, height=0.7, t_end=0.02, cfl=0.45, alpha=ALPHA, gamma=GAMMA, strategy=strategy)
    R, rsteps, rt = oracle.solve(U, max_steps=15, **kw)
    for blocks in (1, 3):
        V, steps, t, bad = kernel_solve(kh, U, kw, blocks, 15)
        assert (steps, t, bad) == (rsteps, rt, 0), blocks
        assert np.array_equal(V, R, equal_nan=True), blocks


@pytest.mark.parametrize("strategy", range(7))
def test_residual_build_follows_fp64_closer_than_fp32(kh_fast, pkg, oracle, strategy):
    """The FP32 build with residual planes (PackedResidual: FP32 slopes and
    fluxes, the update in FP64 on hi + lo, the result split into the FP32
    and 16-bit residual planes) through the single-problem kernels: after
    15 steps its density is closer to the FP64 build's than the FP32
    build's is, and its ring cells hold FP32 values exactly (the ghost
    kernel zeroes their residuals).  Measured: 2.5e-9 to 3.1e-8 against
    3.2e-8 to 9.0e-8 (relative L1) over the seven presets."""
    nx, ny = 41, 30
    U = pkg.scenarios.seeded_four_quadrant(nx, ny, 60 + strategy)
    if strategy in (5, 6):
        U = oracle.ghost(U, strategy)
    kw = dict(width=1.0, height=0.7, t_end=0.02, cfl=0.45, alpha=ALPHA, gamma=GAMMA, strategy=strategy)
    R = build_solve(kh_fast, 0, U, kw, 3, 15)
    F32 = build_solve(kh_fast, 1, U, kw, 3, 15)
    V = build_solve(kh_fast, 2, U, kw, 3, 15)
    assert V[1] == R[1] and abs(V[2] - R[2]) <= 1e-6 * R[2]
    inner = (slice(2, ny - 2), slice(2, nx - 2), 0)

    def rel(A):
        return np.abs(A[0][inner] - R[0][inner]).sum() / np.abs(R[0][inner]).sum()

    print("preset", strategy, "FP32 with residuals", rel(V), "FP32", rel(F32))
    assert rel(V) <= 1e-7 and rel(V) <= 0.7 * rel(F32), (rel(V), rel(F32))
    ring = np.ones((ny, nx), bool)
    ring[2:-2, 2:-2] = False
    assert np.array_equal(V[0][ring], V[0][ring].astype(np.float32).astype(np.float64))


def test_health_record_names_the_first_bad_step(kh, pkg):
    """A negative pressure planted in an interior cell is reported as step 1;
    the run goes on, as the reference's does."""
    nx, ny = 41, 30
    U = np.ascontiguousarray(pkg.scenarios.seeded_four_quadrant(nx, ny, 3)[..., :4])
    kw = dict(width=1.0, height=0.7, t_end=1.0, cfl=0.45, alpha=ALPHA, gamma=GAMMA, strategy=0)
    assert kernel_solve(kh, U, kw, 2, 3)[3] == 0
    U[12, 17, 1] = -1.0
    V, steps, _, bad = kernel_solve(kh, U, kw, 2, 3)
    assert bad == 1 and steps == 3


@pytest.mark.parametrize("nx,ny,blocks", [(64, 48, 1), (200, 120, 4), (37, 5, 3)])
def test_frames_match_a_numpy_rendering(kh, pkg, tmp_path, nx, ny, blocks):
    from test_frames_gpu import read_png, render

    U = np.ascontiguousarray(pkg.scenarios.seeded_four_quadrant(nx, ny, 8)[..., :4])
    U[..., 0] *= 1.0 + 0.01 * np.sin(np.arange(nx))[None, :]  # more than four density values
    path = str(tmp_path / "f.png")
    assert kh.kh_frame(U.ctypes.data, nx, ny, blocks, path.encode()) == 0
    img = read_png(path)  # checks the chunk CRCs and, through zlib, the Adler-32
    want = render(U[..., 0])
    d = np.abs(img.astype(int) - want.astype(int))
    assert img.shape == (ny, nx, 3)
    assert d.max() <= 3 and (d == 0).mean() > 0.99  # a level can differ at a rounding tie
    if 3 * nx * ny + ny > 65535:  # several stored blocks
        assert os.path.getsize(path) > 65535


def test_frame_of_a_uniform_density(kh, tmp_path):
    U = np.ones((20, 30, 4))
    path = str(tmp_path / "u.png")
    assert kh.kh_frame(U.ctypes.data, 30, 20, 2, path.encode()) == 0
    from test_frames_gpu import read_png

    img = read_png(path)
    assert np.all(img == img[0, 0]) and tuple(img[0, 0]) == (68, 1, 84)  # level 0: the first viridis stop


@pytest.mark.parametrize("strategy", range(7))
def test_fp32_adjoint_kernels_agree_with_fp64(kh, k32, oracle, pkg, strategy):
    """The FP32 build's VJP of one step (its taped FP32 forward, the adjoint
    kernels in single precision) against the FP64 one on FP32 values:
    measured 1.1e-7 to 4.1e-6 relative L2; a limiter choice that flips
    between the FP32 and FP64 forward states may add more in a few cells."""
    nx, ny, width, height, t = 37, 29, 1.0, 0.8, 0.01
    U, dt, rng = adjoint_case(oracle, pkg, strategy)
    U = np.ascontiguousarray(U.astype(np.float32).astype(np.float64))
    w = np.ascontiguousarray(rng.standard_normal(U.shape).astype(np.float32).astype(np.float64))
    g64, g32 = np.empty_like(U), np.empty_like(U)
    args = (nx, ny, strategy, t, dt, width, height, ALPHA, GAMMA, 8)
    assert kh.kh_step_vjp(U.ctypes.data, w.ctypes.data, *args, g64.ctypes.data) == 0
    assert k32.k32_step_vjp(U.ctypes.data, w.ctypes.data, *args, g32.ctypes.data) == 0
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel <= 1e-4, rel


@pytest.mark.parametrize("nx,ny,pitch,blocks", [(37, 29, 64, 1), (64, 48, 64, 3), (70, 33, 96, 2)])
def test_conserved_totals_kernels(kh, nx, ny, pitch, blocks):
    """fvm2d_get_conserved_totals' kernels (csrc/fvm2d_transfer.cuh) on the
    host: the interior totals of mass, momenta and energy in FP64 for each
    storage (FP64 planes, FP32 planes, FP32 planes with residuals), against
    exactly summed totals of the values each storage holds; the ghost ring
    (set to huge values here) is left out; the same state gives the same bits."""
    import math
    rng = np.random.default_rng(nx * ny)
    U = np.empty((ny, nx, 4))
    U[..., 0] = rng.uniform(0.1, 2.0, (ny, nx))
    U[..., 1] = rng.uniform(0.02, 2.0, (ny, nx))
    U[..., 2:] = rng.uniform(-1.5, 1.5, (ny, nx, 2))
    ring = np.ones((ny, nx), bool)
    ring[2:-2, 2:-2] = False
    U[ring] = 1e30
    gamma, area = 1.4, 0.37

    def held(storage):  # the values the storage keeps, as FP64
        if storage == 0:
            return U
        if storage == 1:
            return U.astype(np.float32).astype(np.float64)
        hi = U.astype(np.float32).astype(np.float64)
        lo = (U - hi).astype(np.float32)  # rounded to nearest; the kernel cuts toward zero to bfloat16
        return hi + lo.astype(np.float64)  # within 2^-31 relative of U either way

    for storage in (0, 1, 2):
        out = np.empty(4)
        assert kh.kh_totals(np.ascontiguousarray(U).ctypes.data, nx, ny, pitch, storage, blocks, gamma, area,
                            out.ctypes.data) == 0
        V = held(storage)[2:-2, 2:-2]
        r, p, u, v = V[..., 0], V[..., 1], V[..., 2], V[..., 3]
        exact = np.array([math.fsum(x.ravel()) for x in
                          (r, r * u, r * v, p / (gamma - 1) + 0.5 * r * (u * u + v * v))]) * area
        scale = np.array([math.fsum(np.abs(x).ravel()) for x in (r, r * u, r * v, r)]) * area
        tol = 1e-14 if storage < 2 else 1e-9
        assert np.all(np.abs(out - exact) <= tol * scale), (storage, out, exact)
        again = np.empty(4)
        kh.kh_totals(np.ascontiguousarray(U).ctypes.data, nx, ny, pitch, storage, blocks, gamma, area,
                     again.ctypes.data)
        assert np.array_equal(out, again)
