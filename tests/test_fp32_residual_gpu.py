"""FP32 build with residual planes (FVM2D_FP32_RESIDUAL): FP32 slopes, GRP and
fluxes from the FP32 plane values; each stored value kept as an FP32 value
plus a 16-bit (bfloat16) residual; the conservative update of a cell in FP64
from hi + lo, split back into the two planes.

* Density within relative L1 1e-5 of the FP64 path on the four-quadrant
  workload and on the vortex, and closer to it than the FP32 build.
* A state set on the handle reads back as hi + lo of each value (the
  storage's own rounding, emulated here in numpy); a state read back and set
  again continues bit for bit; switching precisions keeps the state.
* Rows read and written for a slab's halo carry hi + lo.
* The ring cells hold FP32 values exactly (their residuals are zeroed).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RHO_L1 = 1e-5  # density relative L1 against the FP64 path


def stored(U):
    """The value the residual storage keeps for each double of U: hi = U
    rounded to FP32, plus U - hi rounded toward zero to FP32 and cut to its
    upper 16 bits (bfloat16)."""
    hi = U.astype(np.float32).astype(np.float64)
    r = U - hi
    rf = r.astype(np.float32)
    over = np.abs(rf.astype(np.float64)) > np.abs(r)
    rf[over] = np.nextafter(rf[over], np.float32(0))
    lo = (rf.view(np.uint32) & np.uint32(0xFFFF0000)).view(np.float32)
    return hi + lo.astype(np.float64)


def run(pkg, U0, precision, steps=None, **kw):
    ny, nx = U0.shape[:2]
    h = pkg.Handle(nx, ny)
    try:
        h.configure(kw.get("width", 1.0), kw.get("height", 1.0), kw.get("t_end", 0.0), kw.get("cfl", 0.45),
                    kw.get("alpha", 1.9), kw.get("gamma", 1.4), kw.get("strategy", 0), precision)
        h.set_state(U0)
        if steps is None:
            h.solve()
        else:
            h.advance(steps)
        t, k, _ = h.time()
        return h.get_state(4), k, t
    finally:
        h.close()


def rel_l1(A, B, f=0):
    return np.abs(A[..., f] - B[..., f]).sum() / np.abs(B[..., f]).sum()


def test_quadrant_workload_density_error(pkg):
    """400x400 four-quadrant problem to t = 0.2 (620 FP64 steps)."""
    U0 = pkg.scenarios.seeded_four_quadrant(400, 400, 0)
    kw = dict(t_end=0.2, cfl=0.45, alpha=1.9, strategy=0)
    D, kd, td = run(pkg, U0, pkg.FP64, **kw)
    S, ks, ts = run(pkg, U0, pkg.FP32, **kw)
    R, kr, tr = run(pkg, U0, pkg.FP32_RESIDUAL, **kw)
    assert tr == pytest.approx(td, abs=1e-12)
    assert abs(kr - kd) <= 2
    err, err32 = rel_l1(R, D), rel_l1(S, D)
    print("four-quadrant 400^2: FP32 with residuals", err, "FP32", err32)
    assert err <= RHO_L1 and err < err32, (err, err32)


def test_vortex_density_error(pkg):
    """Isentropic vortex on periodic [0,10]^2 (256^2 interior), a tenth of a
    period."""
    n = 260
    width, height, _ = pkg.scenarios.periodic_square_layout(n)
    U0 = pkg.scenarios.isentropic_vortex(n)
    kw = dict(width=width, height=height, t_end=1.0, cfl=0.45, alpha=1.9, strategy=5)
    D, _, _ = run(pkg, U0, pkg.FP64, **kw)
    S, _, _ = run(pkg, U0, pkg.FP32, **kw)
    R, _, _ = run(pkg, U0, pkg.FP32_RESIDUAL, **kw)
    inner = (slice(2, n - 2), slice(2, n - 2))
    err, err32 = rel_l1(R[inner], D[inner]), rel_l1(S[inner], D[inner])
    print("vortex 260^2: FP32 with residuals", err, "FP32", err32)
    assert err <= RHO_L1 and err < err32, (err, err32)


def test_state_reads_back_as_stored_and_resumes_bit_for_bit(pkg):
    nx, ny = 203, 150  # rows not a multiple of 32
    U0 = pkg.scenarios.seeded_four_quadrant(nx, ny, 9)[..., :4]
    U0 = U0 * (1.0 + 1e-3 * np.sin(np.arange(nx * ny * 4)).reshape(U0.shape))  # values with residuals
    h = pkg.Handle(nx, ny)
    h.configure(t_end=1.0, precision=pkg.FP32_RESIDUAL)
    h.set_state(U0)
    S = h.get_state(4)
    assert np.array_equal(S, stored(U0))
    assert np.abs(S - U0).max() <= 2.0 ** -31 * np.abs(U0).max()
    h.advance(5)
    mid = h.get_state(4)
    h2 = pkg.Handle(nx, ny)
    h2.configure(t_end=1.0, precision=pkg.FP32_RESIDUAL)
    h2.set_state(mid)
    assert np.array_equal(h2.get_state(4), mid)  # hi + lo splits back into the same hi and lo
    h.advance(5)
    h2.advance(5)
    assert np.array_equal(h.get_state(4), h2.get_state(4))
    # the ring cells hold FP32 values exactly
    V = h.get_state(4)
    ring = np.ones((ny, nx), bool)
    ring[2:-2, 2:-2] = False
    assert np.array_equal(V[ring], V[ring].astype(np.float32).astype(np.float64))
    h.close()
    h2.close()


def test_precision_switch_keeps_the_state(pkg):
    U0 = pkg.scenarios.seeded_four_quadrant(64, 48, 5)[..., :4]
    U0 = U0 * (1.0 + 1e-3 * np.cos(np.arange(64 * 48 * 4)).reshape(U0.shape))
    h = pkg.Handle(64, 48)
    h.configure(t_end=1.0)
    h.set_state(U0)
    h.configure(t_end=1.0, precision=pkg.FP32_RESIDUAL)
    S = h.get_state(4)
    assert np.array_equal(S, stored(U0))
    h.advance(3)
    S3 = h.get_state(4)
    h.configure(t_end=1.0, precision=pkg.FP64)
    assert np.array_equal(h.get_state(4), S3)  # hi + lo is exact in FP64
    h.configure(t_end=1.0, precision=pkg.FP32)
    assert np.array_equal(h.get_state(4), S3.astype(np.float32).astype(np.float64))
    h.configure(t_end=1.0, precision=pkg.FP32_RESIDUAL)
    h.advance(3)
    assert h.time()[1] == 6
    h.close()


def test_rows_carry_the_residuals(pkg):
    nx, ny = 96, 40
    U0 = pkg.scenarios.seeded_four_quadrant(nx, ny, 4)[..., :4]
    U0 = U0 * (1.0 + 1e-3 * np.sin(np.arange(nx * ny * 4)).reshape(U0.shape))
    h = pkg.Handle(nx, ny)
    h.configure(t_end=1.0, precision=pkg.FP32_RESIDUAL)
    h.set_state(U0)
    rows = h.get_rows(10, 3)
    assert np.array_equal(rows, np.moveaxis(stored(U0)[10:13], 2, 0))
    h.set_rows(20, rows)
    assert np.array_equal(h.get_state(4)[20:23], stored(U0)[10:13])
    h.close()
