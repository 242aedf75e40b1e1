"""Initial-data helpers restate the reference's demo initializers (test2D.cu:4-133)."""
import math

import numpy as np


def test_shapes(pkg):
    sc = pkg.scenarios
    assert sc.double_mach(12).shape == (12, 48, 4)
    assert sc.jet(10).shape == (10, 20, 4)
    assert sc.jet800(10).shape == (10, 30, 4)
    assert sc.four_shocks(20).shape == (20, 20, 4)
    assert sc.four_contacts(20).shape == (20, 20, 4)
    assert sc.sedov_1d(16).shape == (16, 16, 4)


def test_double_mach_front(pkg):
    U = pkg.scenarios.double_mach(12)
    for i in range(12):
        l = 12 // 6 + int((12 - i + 3) / math.sqrt(3))
        assert np.all(U[i, :l, 0] == 8.0) and np.all(U[i, l:, 0] == 1.4)


def test_quadrants(pkg):
    U = pkg.scenarios.four_quadrant((1, 1, 1, 1), (2, 2, 2, 2), (3, 3, 3, 3), (4, 4, 4, 4), 6, 4)
    assert U[0, 0, 0] == 2 and U[0, 5, 0] == 1 and U[3, 0, 0] == 3 and U[3, 5, 0] == 4
    V = pkg.scenarios.seeded_four_quadrant(8, 8, 5)
    assert np.all((V[..., 0] >= 0.1) & (V[..., 0] <= 2.0))
    assert np.all((V[..., 1] >= 0.02) & (V[..., 1] <= 2.0))
    assert np.all(np.abs(V[..., 2:]) <= 1.5)


def test_sedov(pkg):
    U = pkg.scenarios.sedov_1d(16)
    assert U[3, 8, 1] == 0.4 * 3200000.0 / (8.0 / 16) and U[3, 7, 1] == U[3, 8, 1]
    assert U[3, 6, 1] == 0.4 * 1e-12


def test_stacked_tiles_built_row_range_by_row_range(pkg):
    sc = pkg.scenarios
    A = np.concatenate([sc.seeded_four_quadrant(40, 30, k) for k in range(3)])
    for lo, hi in [(0, 90), (5, 37), (28, 32), (29, 61), (60, 90), (0, 1), (89, 90), (15, 16)]:
        assert np.array_equal(sc.stacked_four_quadrant_rows(40, 30, lo, hi), A[lo:hi]), (lo, hi)
