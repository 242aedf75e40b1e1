"""Conserved totals (fvm2d_get_conserved_totals): mass, x momentum, y momentum
and energy of the interior cells, computed on the device in FP64 whatever the
precision of the state.

* They equal the totals of the state read back, summed exactly on the host,
  in every precision build, and a second call gives the same bits.
* On a periodic problem the split step keeps the mass: to rounding in FP64
  and with residual planes, to the FP32 storage's rounding in FP32.
* The totals can be written to device memory.
"""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECISIONS = ("FP64", "FP32", "FP32_RESIDUAL")


def exact_totals(U, gamma, area):
    V = U[2:-2, 2:-2]
    r, p, u, v = V[..., 0], V[..., 1], V[..., 2], V[..., 3]
    parts = (r, r * u, r * v, p / (gamma - 1) + 0.5 * r * (u * u + v * v))
    return (np.array([math.fsum(x.ravel()) for x in parts]) * area,
            np.array([math.fsum(np.abs(x).ravel()) for x in parts]) * area)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_totals_equal_the_state_summed_exactly(pkg, precision):
    nx, ny, width, height, gamma = 150, 97, 1.5, 0.97, 1.4
    U0 = pkg.scenarios.seeded_four_quadrant(nx, ny, 11)
    h = pkg.Handle(nx, ny)
    try:
        h.configure(width, height, 0.2, 0.45, 1.9, gamma, 0, getattr(pkg, precision))
        h.set_state(U0)
        h.advance(10)
        T = h.conserved_totals()
        again = h.conserved_totals()
        S = h.get_state(4)  # the stored values, exactly, as doubles
    finally:
        h.close()
    exact, scale = exact_totals(S, gamma, (width / nx) * (height / ny))
    # fixed-order FP64 sums of the same values: rounding only
    assert np.all(np.abs(T - exact) <= 1e-13 * scale), (T, exact)
    assert np.array_equal(T, again)


@pytest.mark.parametrize("precision,bound", [("FP64", 1e-13), ("FP32_RESIDUAL", 1e-9), ("FP32", 1e-6)])
def test_mass_is_kept_on_a_periodic_problem(pkg, precision, bound):
    """128^2 periodic vortex with density modes, 40 steps: the interior mass
    changes only by rounding (the conservative update's flux differences and
    the average of the two split orders; FP32 also rounds every stored
    value).  Momentum and energy are reported, not bounded: the average of
    the split orders in primitive variables does not keep them exactly."""
    sc = pkg.scenarios
    n = 128
    w, hgt, _ = sc.periodic_square_layout(n)
    U0 = sc.isentropic_vortex(n, perturbation=sc.density_modes(16, 1e-3, 3))
    h = pkg.Handle(n, n)
    try:
        h.configure(w, hgt, 1e9, 0.45, 1.9, 1.4, 5, getattr(pkg, precision))
        h.set_state(U0)
        a = h.conserved_totals()
        assert h.advance(40) == 40
        b = h.conserved_totals()
    finally:
        h.close()
    drift = np.abs(b - a) / np.abs(a)
    print(precision, "relative change of mass, momenta, energy over 40 steps:", drift)
    assert drift[0] <= bound, drift


def test_totals_to_device_memory(pkg):
    torch = pytest.importorskip("torch")
    import ctypes
    U0 = pkg.scenarios.seeded_four_quadrant(40, 30, 9)
    h = pkg.Handle(40, 30)
    try:
        h.configure(t_end=0.01, cfl=0.45)
        h.set_state(U0)
        host = h.conserved_totals()
        dev = torch.zeros(4, dtype=torch.float64, device="cuda")
        rc = h.lib.fvm2d_get_conserved_totals(h.h, ctypes.cast(dev.data_ptr(), ctypes.POINTER(ctypes.c_double)))
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(dev.cpu().numpy(), host)
    finally:
        h.close()
