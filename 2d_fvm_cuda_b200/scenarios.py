"""Initial data for the solver: the reference's demo scenarios and seeded workloads.

Every function returns a float64 array of shape (ny, nx, 4) holding the
primitive fields (rho, p, u, v) row-major, row j = 0 at the top of the
domain, the two outer layers on each side being ghost cells -- the layout
RGRP_2D_CUDA takes (src/wrappers.cuh:67-78 flattens rows the same way).

Axis convention (from the reference's direction swap, src/basicFuns.cuh:249-262):
+u points to increasing column i, +v points to DECREASING row j, so the
physical coordinate of row j is y = height - (j + 1/2) * height / ny.
"""
from __future__ import annotations

import math

import numpy as np

POST_SHOCK_2MACH = (8.0, 116.5, 4.125 * math.sqrt(3.0), -4.125)
PRE_SHOCK_2MACH = (1.4, 1.0, 0.0, 0.0)


def four_quadrant(U1, U2, U3, U4, nx: int, ny: int) -> np.ndarray:
    """Four constant states split at (nx/2, ny/2): U2 | U1 over U3 | U4
    (src/wrappers.cuh:80-108, RGRP_2D_CUDA::setRPInitialData)."""
    U = np.empty((ny, nx, 4))
    hx, hy = nx // 2, ny // 2
    U[:hy, :hx] = U2[:4]
    U[hy:, :hx] = U3[:4]
    U[:hy, hx:] = U1[:4]
    U[hy:, hx:] = U4[:4]
    return U


def seeded_quadrant_states(seed: int):
    """Four primitive states rho~U[0.1,2], p~U[0.02,2], u,v~U[-1.5,1.5]
    (the four-quadrant workload's distribution), drawn from one seed."""
    r = np.random.default_rng(seed)
    out = []
    for _ in range(4):
        rho = r.uniform(0.1, 2.0)
        p = r.uniform(0.02, 2.0)
        u = r.uniform(-1.5, 1.5)
        v = r.uniform(-1.5, 1.5)
        out.append((rho, p, u, v))
    return out


def seeded_four_quadrant(nx: int, ny: int, seed: int) -> np.ndarray:
    """The seeded four-quadrant Riemann problem split at the domain centre."""
    return four_quadrant(*seeded_quadrant_states(seed), nx, ny)


def double_mach(n: int) -> np.ndarray:
    """Double Mach reflection, n rows x 4n columns (test2D.cu:4-18)."""
    U = np.empty((n, 4 * n, 4))
    U[:] = PRE_SHOCK_2MACH
    for i in range(n - 1, -1, -1):
        temp = float(n - i + 3) / math.sqrt(3.0)
        length = n // 6 + int(temp)
        U[i, :length] = POST_SHOCK_2MACH
    return U


def jet(n: int) -> np.ndarray:
    """Mach-800-speed jet entering at the left, n rows x 2n columns (test2D.cu:20-31)."""
    U = np.empty((n, 2 * n, 4))
    U[:] = (0.5, 0.4127, 0.0, 0.0)
    for i in range(n):
        if 2 * n // 5 + 1 <= i <= 3 * n // 5:
            U[i, 0] = (5.0, 0.4127, 800.0, 0.0)
    return U


def jet800(n: int) -> np.ndarray:
    """Jet along the bottom wall, n rows x 3n columns (test2D.cu:33-44)."""
    U = np.empty((n, 3 * n, 4))
    U[:] = (0.14, 1.0, 0.0, 0.0)
    for i in range(n):
        if i > 9 * n // 10:
            U[i, 0] = (1.4, 1.0, 800.0, 0.0)
    return U


def four_shocks(n: int) -> np.ndarray:
    """Four-shock Riemann problem split at (4n/5, n/5), n x n (test2D.cu:46-80)."""
    U1 = (1.5, 1.5, 0.0, 0.0)
    U2 = (0.5323, 0.3, 1.206, 0.0)
    U3 = (0.138, 0.029, 1.206, 1.206)
    U4 = (0.5323, 0.3, 0.0, 1.206)
    U = np.empty((n, n, 4))
    r, c = n // 5, 4 * n // 5
    U[:r, :c] = U2
    U[:r, c:] = U1
    U[r:, :c] = U3
    U[r:, c:] = U4
    return U


def four_contacts(n: int) -> np.ndarray:
    """Four contact discontinuities split at the centre, n x n (test2D.cu:82-116)."""
    U1 = (1.0, 1.0, 0.75, -0.5)
    U2 = (2.0, 1.0, 0.75, 0.5)
    U3 = (1.0, 1.0, -0.75, 0.5)
    U4 = (3.0, 1.0, -0.75, -0.5)
    U = np.empty((n, n, 4))
    h = n // 2
    U[:h, :h] = U2
    U[:h, h:] = U1
    U[h:, :h] = U3
    U[h:, h:] = U4
    return U


def sedov_1d(n: int) -> np.ndarray:
    """Planar Sedov blast: two high-pressure columns at the centre, n x n (test2D.cu:118-133)."""
    E0 = 3200000.0
    domain_size = 4.0
    dx = 2 * domain_size / n
    U = np.empty((n, n, 4))
    U[:] = (1.0, 0.4 * 1e-12, 0.0, 0.0)
    U[:, n // 2] = (1.0, 0.4 * E0 / dx, 0.0, 0.0)
    U[:, n // 2 - 1] = (1.0, 0.4 * E0 / dx, 0.0, 0.0)
    return U
