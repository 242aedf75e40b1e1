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


def four_quadrant(U1, U2, U3, U4, nx: int, ny: int, split=None) -> np.ndarray:
    """Four constant states split at (nx/2, ny/2): U2 | U1 over U3 | U4
    (src/wrappers.cuh:80-108, RGRP_2D_CUDA::setRPInitialData).  `split`
    (fractions (sx, sy) of the width and height, measured from the left and
    from the top row) moves the split point."""
    U = np.empty((ny, nx, 4))
    hx, hy = nx // 2, ny // 2
    if split is not None:
        hx, hy = int(round(split[0] * nx)), int(round(split[1] * ny))
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


def seeded_four_quadrant(nx: int, ny: int, seed: int, split=None) -> np.ndarray:
    """The seeded four-quadrant Riemann problem split at the domain centre (or
    at `split`, see four_quadrant)."""
    return four_quadrant(*seeded_quadrant_states(seed), nx, ny, split)


def stacked_four_quadrant_rows(nx: int, tile_ny: int, lo: int, hi: int) -> np.ndarray:
    """Rows [lo, hi) of seeded four-quadrant tiles of tile_ny rows stacked
    top to bottom, tile k drawn from seed k (tile k alone is
    seeded_four_quadrant(nx, tile_ny, k)): one tall problem whose rows can be
    built slab by slab without the whole array."""
    U = np.empty((hi - lo, nx, 4))
    hx = nx // 2
    for k in range(lo // tile_ny, (hi - 1) // tile_ny + 1):
        U1, U2, U3, U4 = seeded_quadrant_states(k)
        a, b = max(lo, k * tile_ny), min(hi, (k + 1) * tile_ny)
        mid = k * tile_ny + tile_ny // 2
        top = slice(a - lo, max(a, min(b, mid)) - lo)
        bot = slice(max(a, min(b, mid)) - lo, b - lo)
        U[top, :hx], U[top, hx:] = U2[:4], U1[:4]
        U[bot, :hx], U[bot, hx:] = U3[:4], U4[:4]
    return U


def uneven_batch(count: int, seed: int, sizes=tuple(range(128, 1025, 64))):
    """`count` seeded four-quadrant problems for the batched form: per-side
    size drawn from `sizes`, split point ~U[0.3, 0.7]^2, states as
    seeded_quadrant_states.  Returns a list of (nx, ny, seed, split)."""
    r = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(r.choice(sizes))
        split = (float(r.uniform(0.3, 0.7)), float(r.uniform(0.3, 0.7)))
        out.append((n, n, int(r.integers(0, 2 ** 31 - 1)), split))
    return out


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


# ---------------------------------------------------------------------------
# Smooth and shock-interface workloads (no reference counterpart: they use the
# periodic and reflective-wall presets this solver adds).
# ---------------------------------------------------------------------------
_GL3 = (np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)]) / 2.0, np.array([5.0, 8.0, 5.0]) / 18.0)


def _prim_from_cons(rho, mx, my, E, gamma):
    u, v = mx / rho, my / rho
    return np.stack([rho, (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v)), u, v], axis=-1)


def vortex_point(x, y, t=0.0, L=10.0, eps=5.0, xc=5.0, yc=5.0, gamma=1.4, u0=1.0, v0=1.0):
    """Isentropic vortex (Shu) translated with the background (rho, u, v, p) =
    (1, u0, v0, 1) on the periodic square [0, L]^2.  Returns conserved
    (rho, rho u, rho v, E) at the points (x, y)."""
    dx = np.mod(x - xc - u0 * t + L / 2, L) - L / 2
    dy = np.mod(y - yc - v0 * t + L / 2, L) - L / 2
    r2 = dx * dx + dy * dy
    f = np.exp(0.5 * (1.0 - r2))
    u = u0 - eps / (2 * np.pi) * f * dy
    v = v0 + eps / (2 * np.pi) * f * dx
    T = 1.0 - (gamma - 1.0) * eps * eps / (8 * gamma * np.pi ** 2) * f * f
    rho = T ** (1.0 / (gamma - 1.0))
    p = rho * T
    return rho, rho * u, rho * v, p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)


def periodic_square_layout(n: int, L: float = 10.0):
    """(width, height, h) for an n x n array whose interior n-4 cells span
    exactly [0, L]: the two ghost layers on each side lie outside."""
    h = L / (n - 4)
    return n * h, n * h, h


def density_modes(count: int, amplitude: float, seed: int, L: float = 10.0, kmax: int = 4):
    """`count` seeded periodic Fourier modes a sin(2 pi kx x / L + p) sin(2 pi ky y / L + q)
    with |a| <= amplitude and 1 <= kx, ky <= kmax; returns a function of (x, y)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(1, kmax + 1, size=(count, 2))
    a = rng.uniform(-amplitude, amplitude, size=count)
    ph = rng.uniform(0.0, 2 * np.pi, size=(count, 2))

    def f(x, y):
        out = np.zeros(np.broadcast(x, y).shape)
        for m in range(count):
            out += a[m] * np.sin(2 * np.pi * k[m, 0] * x / L + ph[m, 0]) * np.sin(2 * np.pi * k[m, 1] * y / L + ph[m, 1])
        return out
    return f


def isentropic_vortex(n: int, t: float = 0.0, L: float = 10.0, eps: float = 5.0, gamma: float = 1.4,
                      perturbation=None) -> np.ndarray:
    """Cell averages (3x3 Gauss points, conserved variables) of the isentropic
    vortex of strength eps centred at (L/2, L/2) on the background
    (rho, u, v, p) = (1, 1, 1, 1), advected to time t, on an n x n array with
    two periodic ghost layers.  `perturbation(x, y)` (optional) is added to the
    density with u, v and p unchanged.  Cell (i, j) is centred at
    x = (i-2+1/2) h, y = L - (j-2+1/2) h, h = L/(n-4) (row 0 on top)."""
    _, _, h = periodic_square_layout(n, L)
    xs = (np.arange(n) - 2 + 0.5) * h
    ys = L - (np.arange(n) - 2 + 0.5) * h
    q, w = _GL3
    acc = np.zeros((4, n, n))
    for a in range(3):
        for b in range(3):
            X = xs[None, :] + q[a] * h
            Y = ys[:, None] + q[b] * h
            rho, mx, my, E = vortex_point(X, Y, t, L, eps, L / 2, L / 2, gamma)
            if perturbation is not None:
                u, v = mx / rho, my / rho
                p = (gamma - 1.0) * (E - 0.5 * rho * (u * u + v * v))
                rho = rho + perturbation(X, Y)
                mx, my = rho * u, rho * v
                E = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
            acc += w[a] * w[b] * np.stack([rho, mx, my, E])
    return _prim_from_cons(acc[0], acc[1], acc[2], acc[3], gamma)


def mach2_post_shock(gamma: float = 1.4, rho1: float = 1.0, p1: float = 1.0, mach: float = 2.0):
    """Rankine-Hugoniot state behind a shock of Mach `mach` moving in +x into
    gas at rest (rho1, p1): (rho2, p2, u2)."""
    m2 = mach * mach
    rho2 = rho1 * (gamma + 1.0) * m2 / ((gamma - 1.0) * m2 + 2.0)
    p2 = p1 * (1.0 + 2.0 * gamma / (gamma + 1.0) * (m2 - 1.0))
    s = mach * np.sqrt(gamma * p1 / rho1)
    return rho2, p2, s * (1.0 - rho1 / rho2)


def shock_bubble(nx: int, ny: int, width: float = 2.0, height: float = 1.0, seed: int = 0, gamma: float = 1.4,
                 shock_x: float = 0.1, centre=(0.4, 0.5), radius: float = 0.15, rho_bubble: float = 0.1,
                 modes: int = 8, amplitude: float = 0.01, sub: int = 4) -> np.ndarray:
    """Mach-2 planar shock at x = shock_x moving in +x towards a light
    circular bubble (rho = rho_bubble, p = 1) in gas at rest (rho = 1, p = 1),
    on an nx x ny array spanning [0, width] x [0, height] (ghosts included).
    The bubble radius carries `modes` seeded Fourier modes whose amplitudes sum
    to at most `amplitude` (relative).  Cells cut by the bubble edge get the
    sub x sub sub-sample average of the two states (conserved variables)."""
    rng = np.random.default_rng(seed)
    a = rng.uniform(0.0, amplitude / modes, modes)
    ph = rng.uniform(0.0, 2 * np.pi, modes)
    rho2, p2, u2 = mach2_post_shock(gamma)
    hx, hy = width / nx, height / ny
    xs = (np.arange(nx) + 0.5) * hx
    ys = height - (np.arange(ny) + 0.5) * hy
    offs = (np.arange(sub) + 0.5) / sub - 0.5
    # cells whose every sub-sample lies on one side of the perturbed edge
    # (radius within radius (1 +- amplitude)) are 0 or 1; only the band between
    # is sub-sampled
    d = np.hypot(xs[None, :] - centre[0], ys[:, None] - centre[1])
    reach = hx + hy
    frac = (d + reach < radius * (1.0 - amplitude)).astype(np.float64)
    jb, ib = np.nonzero((d + reach >= radius * (1.0 - amplitude)) & (d - reach <= radius * (1.0 + amplitude)))
    count = np.zeros(jb.size)
    for ox in offs:
        for oy in offs:
            dx, dy = xs[ib] + ox * hx - centre[0], ys[jb] + oy * hy - centre[1]
            th = np.arctan2(dy, dx)
            r = radius * (1.0 + sum(a[k] * np.cos((k + 1) * th + ph[k]) for k in range(modes)))
            count += (dx * dx + dy * dy < r * r)
    frac[jb, ib] = count / (sub * sub)
    U = np.empty((ny, nx, 4))
    U[..., 0] = rho_bubble * frac + 1.0 * (1.0 - frac)
    U[..., 1] = 1.0
    U[..., 2] = 0.0
    U[..., 3] = 0.0
    post = xs[None, :] < shock_x
    U[..., 0] = np.where(post, rho2, U[..., 0])
    U[..., 1] = np.where(post, p2, U[..., 1])
    U[..., 2] = np.where(post, u2, U[..., 2])
    return U
