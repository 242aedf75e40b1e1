"""The sweep kernels' arithmetic policies checked against one another on the
host (no GPU): tests/math_host.cpp compiles 2d_fvm_cuda_b200/csrc/
fvm2d_math.cuh with g++ (contraction off) and exposes the relaxation GRP,
the interface flux, the conservative update and the limited slopes of each
policy.

* Hoisted (the FP64 product build's shared reciprocals: 4 divisions and 2
  reciprocal square roots per interface) equals RefOrder (the reference's
  expressions and order, src/basicFuns.cuh:37-246) to rounding, in every wave
  case of the GRP: the whole fan to the right, to the left, and the star
  region on either side of the contact.
* The same policy in single precision stays within FP32 rounding of the
  double-precision reference order, and the compensated update
  (HoistedCompensated) is more accurate than the plain one; the FP32
  build's packed form of it (PackedCompensated, two-wide FP32 operations)
  gives the same results as the scalar form.
* The slope limiter on raw differences picks exactly the reference's zero
  pattern.
* The operations each policy spends per interface, counted per wave case
  with a counting number type: the shared-reciprocal form's 4 divisions and
  2 reciprocal square roots (3 and 2 when the fan is one-sided) against the
  reference expressions' 61 divisions by a variable and 4 square roots.
* The hand-written adjoint that the VJP kernels run (interface flux, update,
  limiter; csrc/fvm2d_adjoint_math.cuh) is the transpose of the forward's
  tangent: per interface, <J v, w> = <v, J^T w> with J v from dual numbers
  through Hoisted, and the dual-number tangent matches central differences.

Tolerances are normwise per component (errors divided by |value| plus the
component's median magnitude), with the values measured on x86-64 in the
comments.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CUDA_INC = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
H, DT, GAMMA, ALPHA = 1 / 400, 0.4 / 400 / 8, 1.4, 1.9
K4 = (H, DT, GAMMA, ALPHA)


@pytest.fixture(scope="module")
def mh(tmp_path_factory):
    if shutil.which("g++") is None or not os.path.exists(os.path.join(CUDA_INC, "cuda_runtime.h")):
        pytest.skip("needs g++ and the CUDA headers")
    so = str(tmp_path_factory.mktemp("math_host") / "libmath_host.so")
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-shared", "-fPIC", "-I", CUDA_INC,
                    os.path.join(HERE, "math_host.cpp"), "-o", so], check=True)
    lib = ctypes.CDLL(so)
    for f in ("mh_grp", "mh_flux", "mh_update", "mh_slope"):
        getattr(lib, f).argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
                                    ctypes.c_void_p]
        getattr(lib, f).restype = ctypes.c_int
    lib.mh_count.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.mh_count.restype = ctypes.c_int

    def count(policy, what, x, k4=K4):
        x = np.ascontiguousarray(x, dtype=np.float64)
        k = np.asarray(k4, dtype=np.float64)
        c = np.zeros(8, dtype=np.int64)
        assert lib.mh_count(policy, what, x.ctypes.data, k.ctypes.data, c.ctypes.data) == 0
        return dict(zip(("add", "mul", "div", "div2", "sqrt", "rsqrt", "fma", "cmp"), c.tolist()))

    for f in ("mh_flux_jvp", "mh_flux_vjp", "mh_update_jvp", "mh_update_vjp", "mh_slope_jvp", "mh_slope_vjp"):
        getattr(lib, f).argtypes = [ctypes.c_long] + [ctypes.c_void_p] * 4
        getattr(lib, f).restype = ctypes.c_int

    def call(name, policy, bits, X, k4=K4):
        X = np.ascontiguousarray(X, dtype=np.float64)
        k = np.asarray(k4, dtype=np.float64)
        width = {"mh_grp": 10}.get(name, 4)
        out = np.empty((X.shape[0], width))
        assert getattr(lib, name)(policy, bits, X.shape[0], X.ctypes.data, k.ctypes.data, out.ctypes.data) == 0
        return out

    def deriv(name, X, D, width, k4=K4):
        """name_jvp(X, D = direction) or name_vjp(X, D = output adjoint)."""
        X = np.ascontiguousarray(X, dtype=np.float64)
        D = np.ascontiguousarray(D, dtype=np.float64)
        k = np.asarray(k4, dtype=np.float64)
        out = np.empty((X.shape[0], width))
        assert getattr(lib, name)(X.shape[0], X.ctypes.data, D.ctypes.data, k.ctypes.data, out.ctypes.data) == 0
        return out

    call.deriv = deriv
    call.count = count
    call.lib = lib
    return call


REF, HOISTED, COMPENSATED, PACKED = 0, 1, 2, 3


def cells(rng, n):
    """rho in [0.1, 3] and p in [0.05, 5] (log-uniform), u in [-4, 4],
    v in [-2, 2]: sub- and supersonic states with pressure ratios up to 100."""
    rho = np.exp(rng.uniform(np.log(0.1), np.log(3.0), n))
    p = np.exp(rng.uniform(np.log(0.05), np.log(5.0), n))
    return np.stack([rho, p, rng.uniform(-4, 4, n), rng.uniform(-2, 2, n)], 1)


def interfaces(seed, n=100_000):
    rng = np.random.default_rng(seed)
    L, R = cells(rng, n), cells(rng, n)
    sL = rng.standard_normal((n, 4)) * L * 0.5
    sR = rng.standard_normal((n, 4)) * R * 0.5
    return L, R, np.concatenate([L, R, sL, sR], 1)


def normwise(A, B):
    """max over samples of |A - B| / (|B| + median |B|), per component."""
    return (np.abs(A - B) / (np.abs(B) + np.median(np.abs(B), 0))).max(0)


def test_reference_order_equals_the_oracle(mh, oracle):
    """The host build of RefOrder (what the contraction-free GPU build runs)
    against the oracle's C restatement (oracle/fvm2d_oracle.c, pinned to the
    reference): GRP and slopes bit for bit, so the comparisons of the other
    policies with RefOrder are comparisons with the pinned oracle."""
    _, _, X = interfaces(7, 2000)
    W = mh("mh_grp", REF, 64, X)
    dp = ctypes.POINTER(ctypes.c_double)
    for i in range(len(X)):
        x = [np.ascontiguousarray(X[i, 4 * q:4 * q + 4]) for q in range(4)]
        w, wt = np.zeros(5), np.zeros(5)
        oracle.lib.orc_grp(*[a.ctypes.data_as(dp) for a in x], GAMMA, w.ctypes.data_as(dp), wt.ctypes.data_as(dp))
        assert np.array_equal(W[i], np.concatenate([w, wt]), equal_nan=True), i
    rng = np.random.default_rng(8)
    C = np.concatenate([cells(rng, 2000), cells(rng, 2000), cells(rng, 2000)], 1)
    S = mh("mh_slope", REF, 64, C)
    for i in range(len(C)):
        m, c, p = (np.ascontiguousarray(C[i, 4 * q:4 * q + 4]) for q in range(3))
        s = np.zeros(4)
        oracle.lib.orc_slope(m.ctypes.data_as(dp), c.ctypes.data_as(dp), p.ctypes.data_as(dp), H, ALPHA,
                             s.ctypes.data_as(dp))
        assert np.array_equal(S[i], s), i


def test_hoisted_grp_equals_reference_order_in_every_wave_case(mh):
    L, R, X = interfaces(1)
    W0 = mh("mh_grp", REF, 64, X)
    W1 = mh("mh_grp", HOISTED, 64, X)
    left = (W0[:, 0] == L[:, 0]) & (W0[:, 2] == L[:, 2])
    right = (W0[:, 0] == R[:, 0]) & (W0[:, 2] == R[:, 2])
    star = ~left & ~right
    n = len(X)
    for name, sel in (("fan right", left), ("fan left", right), ("star, u <= 0", star & (W0[:, 2] <= 0)),
                      ("star, u > 0", star & (W0[:, 2] > 0)), ("p_R >= p_L", R[:, 1] >= L[:, 1]),
                      ("p_R < p_L", R[:, 1] < L[:, 1])):
        assert sel.sum() > n // 20, name  # every branch well covered
        e = normwise(W1[sel], W0[sel])
        print(name, sel.sum(), "max normwise", e.max())
        assert e.max() <= 1e-13, (name, e)  # measured 1.9e-14 (the time derivatives)


def wave_cases(W, L, R):
    """0: the fan moves right (left state), 1: left (right state), 2: star
    region with u <= 0, 3: star region with u > 0."""
    left = (W[:, 0] == L[:, 0]) & (W[:, 2] == L[:, 2])
    right = (W[:, 0] == R[:, 0]) & (W[:, 2] == R[:, 2])
    return np.where(left, 0, np.where(right, 1, np.where(W[:, 2] <= 0, 2, 3)))


def test_divisions_and_square_roots_per_interface(mh):
    """Counted per wave case on 2000 interfaces, for the whole interface flux
    (face states, GRP, midpoint flux); counts are the same for every
    interface of a case."""
    L, R, X = interfaces(1, 2000)
    case = wave_cases(mh("mh_grp", REF, 64, X), L, R)
    want = {  # (policy, case): (divisions by a variable, halvings, sqrt, rsqrt)
        (REF, 0): (27, 10, 4, 0), (REF, 1): (28, 10, 4, 0), (REF, 2): (61, 12, 4, 0), (REF, 3): (61, 12, 4, 0),
        (HOISTED, 0): (3, 0, 0, 2), (HOISTED, 1): (3, 0, 0, 2), (HOISTED, 2): (4, 0, 0, 2),
        (HOISTED, 3): (4, 0, 0, 2),
    }
    for c in range(4):
        rows = np.flatnonzero(case == c)
        assert len(rows) > 50, c
        for policy in (REF, HOISTED):
            seen = {tuple(mh.count(policy, 1, X[i])[k] for k in ("div", "div2", "sqrt", "rsqrt")) for i in rows}
            assert seen == {want[(policy, c)]}, (policy, c, seen)


def test_operations_per_cell_and_sweep(mh):
    """A cell's share of one sweep: one interface flux, four limited slopes,
    one update.  The shared-reciprocal slopes need no division and the
    update one (the reference's five); the compensated update adds
    error-free sums and products but no division, and applies 1/(gamma-1)
    and gamma-1 with their low parts."""
    rng = np.random.default_rng(2)
    n = 500
    M = np.concatenate([cells(rng, n), cells(rng, n), cells(rng, n)], 1)
    X = update_inputs(3, n)
    pad = lambda x: np.pad(x, (0, 16 - len(x)))  # noqa: E731
    for i in range(n):
        s0, s1 = mh.count(REF, 2, pad(M[i])), mh.count(HOISTED, 2, pad(M[i]))
        assert s0["div"] == s1["div"] == 0 and s1["mul"] <= s0["mul"]
        u0, u1, u2 = (mh.count(p, 3, pad(X[i])) for p in (REF, HOISTED, COMPENSATED))
        assert (u0["div"], u1["div"], u2["div"]) == (5, 1, 1)
        assert u2["fma"] == 13  # the residuals of the two-products, the gamma constants' low parts


def test_hoisted_flux_equals_reference_order(mh):
    _, _, X = interfaces(2)
    F0 = mh("mh_flux", REF, 64, X)
    F1 = mh("mh_flux", HOISTED, 64, X)
    e = normwise(F1, F0)
    print("flux FP64 normwise", e)
    assert e.max() <= 1e-13, e  # measured 7.2e-15


def test_uniform_state_is_a_fixed_point(mh):
    """Equal face states and zero slopes: the interface state is the cell's
    and every time derivative is zero, in both policies and precisions."""
    rng = np.random.default_rng(3)
    C = cells(rng, 20_000)
    X = np.concatenate([C, C, np.zeros_like(C), np.zeros_like(C)], 1)
    for policy in (REF, HOISTED):
        for bits in (64, 32):
            W = mh("mh_grp", policy, bits, X)
            Cb = C if bits == 64 else C.astype(np.float32).astype(np.float64)
            # the star region recombines u and p from both sides: a few
            # roundings (measured 5.3e-16 in FP64, 2.7e-7 in FP32)
            e = normwise(W[:, :4], Cb)
            assert e.max() <= (4e-15 if bits == 64 else 1e-6), (policy, bits, e)
            assert np.all(W[:, 5:] == 0.0), (policy, bits)


def test_fp32_grp_and_flux_stay_within_single_precision_rounding(mh):
    _, _, X = interfaces(4)
    X32 = X.astype(np.float32).astype(np.float64)  # the FP32 build's inputs
    e = normwise(mh("mh_grp", HOISTED, 32, X32), mh("mh_grp", REF, 64, X32))
    print("grp FP32 vs FP64 normwise", e)
    assert e.max() <= 1e-4, e  # measured 1.3e-5 (energy derivative)
    e = normwise(mh("mh_flux", HOISTED, 32, X32), mh("mh_flux", REF, 64, X32))
    print("flux FP32 vs FP64 normwise", e)
    assert e.max() <= 5e-5, e  # measured 5.4e-6


def update_inputs(seed, n=100_000):
    rng = np.random.default_rng(seed)
    U = cells(rng, n)
    FL = rng.standard_normal((n, 4))
    FR = FL + 0.5 * rng.standard_normal((n, 4))
    # values an FP32 sweep holds: every input exactly representable in FP32
    return np.concatenate([U, FL, FR], 1).astype(np.float32).astype(np.float64)


def update_errors(P, R):
    """Errors of primitives P against R scaled as the conserved variables
    carry them: rho relative, p against (gamma - 1) E, velocities against
    |u| + |v| + sqrt(p / rho)."""
    rho, p, u, v = R.T
    E = p / (GAMMA - 1) + 0.5 * rho * (u * u + v * v)
    vel = np.abs(u) + np.abs(v) + np.sqrt(np.abs(p) / rho)
    return np.stack([np.abs(P[:, 0] - rho) / rho, np.abs(P[:, 1] - p) / ((GAMMA - 1) * E),
                     np.abs(P[:, 2] - u) / vel, np.abs(P[:, 3] - v) / vel], 1)


def test_updates_agree_and_compensation_helps_in_fp32(mh):
    X = update_inputs(5)
    k32 = (float(np.float32(H)), float(np.float32(DT)), GAMMA, ALPHA)  # lambda as the FP32 build forms it
    R0 = mh("mh_update", REF, 64, X, k32)
    ok = (R0[:, 0] > 0) & (R0[:, 1] > 0)
    assert ok.mean() > 0.8
    for policy in (HOISTED, COMPENSATED):
        e = update_errors(mh("mh_update", policy, 64, X, k32), R0)[ok].max(0)
        print("FP64 update policy", policy, e)
        assert e.max() <= 4e-15, (policy, e)  # measured 5.5e-16
    plain = update_errors(mh("mh_update", HOISTED, 32, X, k32), R0)[ok]
    comp = update_errors(mh("mh_update", COMPENSATED, 32, X, k32), R0)[ok]
    print("FP32 plain update: max", plain.max(0), "mean", plain.mean(0))
    print("FP32 compensated update: max", comp.max(0), "mean", comp.mean(0))
    # compensated: about the final rounding to FP32 (measured max 2.9e-7 for
    # rho, 1.1-1.6e-7 for p, u, v; plain: up to 4.1e-7)
    assert comp.max(0)[0] <= 4e-7 and comp.max(0)[1:].max() <= 3e-7, comp.max(0)
    # and smaller on average than the plain FP32 update for p, u and v
    # (measured 0.59, 0.64, 0.63 of it)
    assert np.all(comp.mean(0)[1:] <= 0.8 * plain.mean(0)[1:]), (comp.mean(0), plain.mean(0))


def test_fp32_update_round_trip_keeps_pressure_unbiased(mh):
    """With equal fluxes the update converts p to E and back.  The FP32
    compensated update applies 1/(gamma-1) and gamma-1 with their low parts,
    so the pressure returns without a drift; with the rounded constants
    alone (2.5f and 1.4f - 1) every round trip scaled it by 1 - 6e-8, which
    the tens of thousands of sweeps of a run accumulate."""
    X = update_inputs(7)
    X[:, 8:12] = X[:, 4:8]  # F_R = F_L
    k32 = (float(np.float32(H)), float(np.float32(DT)), GAMMA, ALPHA)
    ok = (X[:, 0] > 0) & (X[:, 1] > 0)
    for policy in (COMPENSATED, PACKED):
        P = mh("mh_update", policy, 32, X, k32)
        rel = (P[ok, 1] - X[ok, 1]) / X[ok, 1]
        print("policy", policy, "p round trip: mean signed", rel.mean(), "max", np.abs(rel).max())
        assert abs(rel.mean()) <= 5e-9, rel.mean()
        assert np.abs(rel).max() <= 3e-7


def test_residual_storage_split(mh):
    """The FP32 build with residual planes keeps x as hi = fl32(x) plus lo =
    x - hi cut toward zero to bfloat16: hi + lo is within 2^-31 |x| of x, x
    halfway between two FP32 values is held exactly, and splitting hi + lo
    again gives the same bits (|lo| stays below half a unit of hi's last
    place), also for remainders just short of that half."""
    rng = np.random.default_rng(8)
    x = rng.standard_normal(200_000) * np.exp(rng.uniform(-20, 20, 200_000))
    hi = rng.standard_normal(20_000).astype(np.float32)
    ulp = np.spacing(np.abs(hi)).astype(np.float64)
    half = np.where(rng.random(20_000) < 0.5, 0.5, -0.5) * ulp
    ties = hi.astype(np.float64) + half
    # remainders just short of half a unit (rounding to nearest would reach it)
    near = hi.astype(np.float64) + half * (1.0 - 2.0 ** -12)
    X = np.concatenate([x, ties, near])
    lib = mh.lib
    lib.mh_split.argtypes = [ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p]
    out = np.empty((len(X), 3))
    assert lib.mh_split(len(X), X.ctypes.data, out.ctypes.data) == 0
    val = out[:, 0] + out[:, 1]
    assert np.all(np.abs(val - X) <= 2.0 ** -31 * np.abs(X)), np.abs(val - X).max()
    assert np.array_equal(val[len(x):len(x) + len(ties)], ties)  # a tie is held exactly
    assert np.all(out[:, 2] == 1.0)


def test_packed_fp32_physics_matches_the_scalar_form(mh):
    """PackedCompensated pairs independent FP32 operations into two-wide
    instructions and regroups a few residual sums; on the host (each pair as
    two correctly rounded operations) it gives the scalar form's results."""
    X = update_inputs(5)
    k32 = (float(np.float32(H)), float(np.float32(DT)), GAMMA, ALPHA)
    P = mh("mh_update", PACKED, 32, X, k32)
    C = mh("mh_update", COMPENSATED, 32, X, k32)
    same = (P == C).all(1).mean()
    print("packed update equal to the scalar compensated update:", same)
    assert same >= 0.999  # measured: all 10^5
    R0 = mh("mh_update", REF, 64, X, k32)
    ok = (R0[:, 0] > 0) & (R0[:, 1] > 0)
    e = update_errors(P, R0)[ok].max(0)
    assert e[0] <= 4e-7 and e[1:].max() <= 3e-7, e
    _, _, XF = interfaces(4)
    XF = XF.astype(np.float32).astype(np.float64)
    F3 = mh("mh_flux", PACKED, 32, XF)
    assert np.array_equal(F3, mh("mh_flux", HOISTED, 32, XF))  # the face states' pairs round alike


def test_hoisted_limiter_picks_the_reference_zero_pattern(mh):
    rng = np.random.default_rng(6)
    n = 100_000
    X = np.concatenate([cells(rng, n), cells(rng, n), cells(rng, n)], 1)
    S0 = mh("mh_slope", REF, 64, X)
    S1 = mh("mh_slope", HOISTED, 64, X)
    nz = S0 != 0
    assert 0.2 < nz.mean() < 0.5
    assert np.array_equal(nz, S1 != 0)
    assert (np.abs(S1 - S0)[nz] / np.abs(S0[nz])).max() <= 1e-15  # measured 2.3e-16
    X32 = X.astype(np.float32).astype(np.float64)
    S0 = mh("mh_slope", REF, 64, X32)
    S1 = mh("mh_slope", HOISTED, 32, X32)
    nz = S0 != 0
    assert np.array_equal(nz, S1 != 0)
    assert (np.abs(S1 - S0)[nz] / np.abs(S0[nz])).max() <= 4e-7  # measured 1.1e-7


def limiter_triples(rng, n):
    """(m, c, p) triples that reach every corner of the limiter: equal
    neighbours, differences at the rounding of the values, subnormal and
    underflowing products, overflowing ones, signed zeros, infinities and
    NaN, besides ordinary data."""
    scale = 10.0 ** rng.uniform(-320, 300, (n, 1))
    X = rng.standard_normal((n, 3)) * scale
    c = rng.uniform(0.1, 3.0, n)
    near = np.stack([c - rng.integers(-3, 4, n) * np.spacing(c), c, c + rng.integers(-3, 4, n) * np.spacing(c)], 1)
    special = np.array([0.0, -0.0, 5e-324, -5e-324, 1e-160, 1e160, np.inf, -np.inf, np.nan, 1.0, -1.0, 2.5])
    S = special[rng.integers(0, len(special), (n, 3))]
    mix = np.where(rng.random((n, 3)) < 0.5, S, X)
    return np.concatenate([X, near, S, mix])


def test_limiter_overloads_equal_the_generic_form(mh):
    """The sweeps' double and float limiters test d1 d2 > 0 alone (d1 d2 > 0
    implies dc d2 > 0) and take the sign of dc by copysign: the same bits as
    the generic form with both tests, on ordinary and degenerate inputs."""
    lib = mh.lib
    lib.mh_limiter_forms.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.mh_limiter_forms.restype = ctypes.c_int
    rng = np.random.default_rng(21)
    X = np.ascontiguousarray(limiter_triples(rng, 200_000))
    for bits, k2 in ((64, (200.0, 380.0)), (64, (0.5, 1.9)), (64, (1e300, 1e-300)), (32, (200.0, 380.0))):
        k = np.asarray(k2, dtype=np.float64)
        out = np.empty((len(X), 2))
        with np.errstate(all="ignore"):
            assert lib.mh_limiter_forms(bits, len(X), X.ctypes.data, k.ctypes.data, out.ctypes.data) == 0
        fast, generic = out[:, 0], out[:, 1]
        if bits == 32:  # the float overload's min instructions differ from selects on NaN arguments only
            with np.errstate(all="ignore"):
                keep = ~np.isnan(X.astype(np.float32)).any(1)
            fast, generic = fast[keep], generic[keep]
        assert np.array_equal(fast.view(np.int64), generic.view(np.int64)), (bits, k2)
        assert (generic != 0).mean() > 0.05


def dot_mismatch(Jv, w, v, JTw):
    """Per row |<Jv, w> - <v, J^T w>| over the sum of the magnitudes of the
    terms of both dot products."""
    a, b = (Jv * w).sum(1), (v * JTw).sum(1)
    return np.abs(a - b) / (np.abs(Jv * w).sum(1) + np.abs(v * JTw).sum(1) + 1e-300)


def test_flux_adjoint_is_the_transpose_of_the_tangent(mh):
    L, R, X = interfaces(8)
    rng = np.random.default_rng(11)
    v = rng.standard_normal(X.shape)
    w = rng.standard_normal((len(X), 4))
    Jv = mh.deriv("mh_flux_jvp", X, v, 4)
    JTw = mh.deriv("mh_flux_vjp", X, w, 16)
    r = dot_mismatch(Jv, w, v, JTw)
    print("flux <Jv,w> vs <v,JTw>: max", r.max())
    # the adjoint recomputes the forward in its own order: rounding only
    assert r.max() <= 1e-12, r.max()  # measured 7.5e-15 over every wave case


def test_flux_tangent_matches_central_differences(mh):
    _, _, X = interfaces(12)
    rng = np.random.default_rng(13)
    v = rng.standard_normal(X.shape) * np.abs(X)  # relative directions
    Jv = mh.deriv("mh_flux_jvp", X, v, 4)
    eps = 1e-6
    fd = (mh("mh_flux", HOISTED, 64, X + eps * v) - mh("mh_flux", HOISTED, 64, X - eps * v)) / (2 * eps)
    r = np.abs(fd - Jv).max(1) / (np.abs(Jv).max(1) + 1e-12)
    print("flux tangent vs central differences: 99.9%", np.quantile(r, 0.999), "max", r.max())
    # differentiable almost everywhere: a sample whose +-eps straddles a
    # wave-case or limiter switch may differ (none in 10^5 at this eps;
    # measured max 2.7e-8)
    assert np.quantile(r, 0.999) <= 1e-7
    assert (r > 1e-4).sum() <= 10


def test_update_adjoint_is_the_transpose_of_the_tangent(mh):
    X = update_inputs(9)
    rng = np.random.default_rng(14)
    v = rng.standard_normal(X.shape)
    w = rng.standard_normal((len(X), 4))
    r = dot_mismatch(mh.deriv("mh_update_jvp", X, v, 4), w, v, mh.deriv("mh_update_vjp", X, w, 12))
    print("update <Jv,w> vs <v,JTw>: max", r.max())
    assert r.max() <= 1e-12, r.max()  # measured 4.7e-15


def test_limiter_adjoint_is_the_transpose_of_the_tangent(mh):
    rng = np.random.default_rng(10)
    n = 100_000
    X = np.concatenate([cells(rng, n), cells(rng, n), cells(rng, n)], 1)
    v = rng.standard_normal(X.shape)
    w = rng.standard_normal((n, 4))
    JTw = mh.deriv("mh_slope_vjp", X, w, 12)
    assert 0.5 < (JTw != 0).any(1).mean() < 0.95  # limited and flat cells both present
    r = dot_mismatch(mh.deriv("mh_slope_jvp", X, v, 4), w, v, JTw)
    print("limiter <Jv,w> vs <v,JTw>: max", r.max())
    assert r.max() <= 1e-14, r.max()  # measured 2.8e-16
