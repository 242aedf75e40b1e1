"""Differentiation form: tangent-linear (fvm2d_jvp) and adjoint (fvm2d_forward +
fvm2d_vjp) of the FP64 step at fixed dt, and the adjoint of the FP32 step
against it.

The scheme is piecewise smooth: the limiter picks one of three differences
or zero, the relaxation speeds take max(0, .), and the Riemann solver has wave
cases.  On a uniform region all of these sit exactly on their switch (equal
face states give a zero argument), where the tangent follows one branch and a
central difference averages two.  Finite differences are therefore taken on
data with no uniform region (large smooth waves in every field) or with
perturbations small against the data's cell-to-cell differences, along smooth
directions, so that only the few cells near an extremum or inflection line
can cross a switch.

* The JVP matches central finite differences of the forward on smooth data.
* Dot-product test: <JVP(v), w> = <v, VJP(w)> for random v, w, over one step
  and over many steps with checkpoints, on every ghost preset.
* The gradient of J = sum (rho_T - rho_target)^2 with respect to the initial
  density (the differentiation workload's objective, on a smaller array)
  matches central finite differences.
* A full-tape forward (every step taped, nothing recomputed in the VJP) gives
  the checkpointed run's state and cotangent, serves several VJPs, and is
  discarded when a parameter changes.
* The checkpointed reverse's two schedules (next segment recomputed on a
  second stream while the current one is reversed, or both in turn on one
  stream) and the full tape give one gradient on every preset.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def vortex_case(pkg, n, seed=3, amp=1e-3):
    sc = pkg.scenarios
    w, h, hh = sc.periodic_square_layout(n)
    U = sc.isentropic_vortex(n, perturbation=sc.density_modes(16, amp, seed))
    return U, w, h, hh


def fixed_dt(pkg, U, hmin, gamma=1.4, cfl=0.45):
    s = np.sqrt(U[..., 2] ** 2 + U[..., 3] ** 2) + np.sqrt(gamma * U[..., 1] / U[..., 0])
    return cfl * hmin / s.max()


def handle(pkg, U, width, height, dt, strategy=5):
    ny, nx = U.shape[:2]
    hd = pkg.Handle(nx, ny)
    hd.configure(width, height, 1e9, 0.45, 1.9, 1.4, strategy, pkg.FP64)
    hd.set_fixed_dt(dt)
    hd.set_state(U)
    return hd


def forward(pkg, U, width, height, dt, steps, strategy=5):
    hd = handle(pkg, U, width, height, dt, strategy)
    hd.advance(steps)
    V = hd.get_state(4)
    hd.close()
    return V


def smooth_direction(pkg, n, seed):
    """A smooth periodic perturbation of all four fields."""
    sc = pkg.scenarios
    _, _, h = sc.periodic_square_layout(n)
    xs = (np.arange(n) - 2 + 0.5) * h
    X, Y = np.meshgrid(xs, 10.0 - xs)
    v = np.zeros((n, n, 4))
    for f in range(4):
        v[..., f] = sc.density_modes(6, 1.0, seed * 10 + f)(X, Y)
    return v


def waves(pkg, n):
    """Periodic state with large smooth waves in every field, varying along both
    directions (no field is uniform along a sweep line)."""
    sc = pkg.scenarios
    w, h, hh = sc.periodic_square_layout(n)
    xs = (np.arange(n) - 2 + 0.5) * hh
    X, Y = np.meshgrid(xs, 10.0 - xs)
    k = 2 * np.pi / 10.0
    U = np.empty((n, n, 4))
    U[..., 0] = 1.0 + 0.3 * np.sin(k * X + 0.3) * np.sin(k * Y + 1.1)
    U[..., 1] = 1.0 + 0.2 * np.cos(k * X + 0.7) * np.sin(2 * k * Y + 0.2)
    U[..., 2] = 0.5 + 0.3 * np.sin(k * Y + 0.4) + 0.2 * np.cos(k * X + 0.9)
    U[..., 3] = -0.3 + 0.2 * np.cos(k * X + 1.3) + 0.15 * np.sin(k * Y + 2.0)
    return U, w, h, hh


def test_jvp_matches_finite_differences(pkg):
    n = 64
    U, w, h, hh = waves(pkg, n)
    dt = fixed_dt(pkg, U, hh)
    v = smooth_direction(pkg, n, 1)
    hd = handle(pkg, U, w, h, dt)
    jv = hd.jvp(10, v)
    hd.close()
    # measured on B200: relative L2 1.6e-8 at eps 1e-8; above it the error
    # grows in proportion to eps (cells pushed across a limiter switch)
    eps = 1e-8
    fd = (forward(pkg, U + eps * v, w, h, dt, 10) - forward(pkg, U - eps * v, w, h, dt, 10)) / (2 * eps)
    err = np.linalg.norm(jv - fd) / np.linalg.norm(fd)
    assert err < 1e-5, err


@pytest.mark.parametrize("strategy", [0, 1, 2, 3, 4, 5, 6])
def test_dot_product_one_step_every_preset(pkg, oracle, strategy):
    n = 48
    U = pkg.scenarios.seeded_four_quadrant(n, 40, 70 + strategy)
    U = oracle.ghost(U, strategy)
    dt = fixed_dt(pkg, U, 1.0 / n) * 0.5
    rng = np.random.default_rng(strategy)
    v = rng.standard_normal(U.shape)
    wv = rng.standard_normal(U.shape)
    hd = handle(pkg, U, 1.0, 40 / n, dt, strategy)
    jv = hd.jvp(1, v)
    hd.set_state(U)
    hd.forward(1, 1)
    vj = hd.vjp(wv)
    hd.close()
    a, b = np.sum(jv * wv), np.sum(v * vj)
    assert abs(a - b) <= 1e-11 * max(abs(a), abs(b)), (a, b)


@pytest.mark.parametrize("steps,checkpoints", [(12, 4), (25, 5), (7, 1), (25, 0)])
def test_dot_product_many_steps_with_checkpoints(pkg, steps, checkpoints):
    U, w, h, hh = vortex_case(pkg, 96)
    dt = fixed_dt(pkg, U, hh)
    rng = np.random.default_rng(steps)
    v = rng.standard_normal(U.shape)
    wv = rng.standard_normal(U.shape)
    hd = handle(pkg, U, w, h, dt)
    jv = hd.jvp(steps, v)
    final_jvp = hd.get_state(4)
    hd.set_state(U)
    hd.forward(steps, checkpoints)
    final = hd.get_state(4)
    # the dual-number build evaluates the same arithmetic in another kernel:
    # both runs end in the same state up to FMA-contraction rounding
    assert np.allclose(final, final_jvp, rtol=1e-12, atol=0)
    vj = hd.vjp(wv)
    assert np.array_equal(hd.get_state(4), final)  # the reverse leaves the final state in place
    hd.close()
    a, b = np.sum(jv * wv), np.sum(v * vj)
    assert abs(a - b) <= 1e-10 * max(abs(a), abs(b)), (a, b)


# Several checkpoint segments, the first one short, on every preset (the
# double-Mach fill depends on the time, so each recomputed segment must start
# from its own checkpoint's time).  The forward tapes its last segment as it
# runs; the VJP recomputes the others on a second stream while reversing
# (overlap on) or in turn on one stream with one tape buffer (overlap off).
# Both schedules, a second VJP of the same forward (which recomputes the
# segment the forward taped) and the full tape (whose forward runs every step
# in order) give one gradient, up to the reordered sums of the ghost
# transpose's atomics.  (The dot-product identity with the JVP is checked on
# smooth data above: over many steps of these discontinuous states the
# dual-number forward, rounded differently, can take another limiter branch.)
@pytest.mark.parametrize("strategy", [0, 1, 2, 3, 4, 5, 6])
def test_checkpoint_schedules_agree_every_preset(pkg, oracle, strategy):
    n, steps, checkpoints = 48, 23, 5  # 5 segments: the first of 3 steps, the others of 5
    U = oracle.ghost(pkg.scenarios.seeded_four_quadrant(n, 40, 110 + strategy), strategy)
    dt = fixed_dt(pkg, U, 1.0 / n) * 0.5
    wv = np.random.default_rng(100 + strategy).standard_normal(U.shape)
    hd = handle(pkg, U, 1.0, 40 / n, dt, strategy)
    grads = []
    for overlap in (True, False):
        hd.set_vjp_overlap(overlap)
        hd.set_state(U)
        hd.forward(steps, checkpoints)
        grads.append(hd.vjp(wv))
        grads.append(hd.vjp(wv))
    hd.set_state(U)
    hd.forward(steps, pkg.FULL_TAPE)
    ref = hd.vjp(wv)
    hd.close()
    for k, g in enumerate(grads):
        rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
        assert rel <= 1e-12, (k, rel)


def test_gradient_of_density_objective_matches_finite_differences(pkg):
    """J = sum (rho_T - rho_target)^2; the gradient with respect to the initial
    density from fvm2d_vjp against central differences along random density
    directions."""
    n, steps = 128, 40
    U, w, h, hh = vortex_case(pkg, n, seed=3)
    Ut, _, _, _ = vortex_case(pkg, n, seed=11)
    dt = fixed_dt(pkg, U, hh)
    target = forward(pkg, Ut, w, h, dt, steps)[..., 0]

    import math

    def J(U0):  # summed accurately: the finite difference cancels most of it
        return math.fsum(((forward(pkg, U0, w, h, dt, steps)[..., 0] - target) ** 2).ravel())

    hd = handle(pkg, U, w, h, dt)
    hd.forward(steps, int(np.ceil(np.sqrt(steps))))
    UT = hd.get_state(4)
    cot = np.zeros_like(U)
    cot[..., 0] = 2 * (UT[..., 0] - target)
    grad = hd.vjp(cot)[..., 0]
    hd.close()
    for k in range(3):
        d = np.zeros_like(U)
        d[..., 0] = smooth_direction(pkg, n, 20 + k)[..., 0]
        eps = 1e-8  # small against the density modes' cell-to-cell differences (~1e-4)
        fd = (J(U + eps * d) - J(U - eps * d)) / (2 * eps)
        ad = np.sum(grad * d[..., 0])
        assert abs(fd - ad) <= 1e-5 * abs(ad), (fd, ad)


def gradient(pkg, U, w, h, dt, steps, target, precision, cot=None):
    """Gradient of J = sum (rho_T - target)^2 with respect to the initial
    density from fvm2d_forward + fvm2d_vjp in `precision`; `cot` replaces the
    cotangent 2 (rho_T - target) of the run's own final state."""
    ny, nx = U.shape[:2]
    hd = pkg.Handle(nx, ny)
    hd.configure(w, h, 1e9, 0.45, 1.9, 1.4, 5, precision)
    hd.set_fixed_dt(dt)
    hd.set_state(U)
    hd.forward(steps, int(np.ceil(np.sqrt(steps))))
    if cot is None:
        UT = hd.get_state(4)
        cot = np.zeros_like(U)
        cot[..., 0] = 2 * (UT[..., 0] - target)
    g = hd.vjp(cot)[..., 0]
    hd.close()
    return g, cot


# FP32 differentiation against FP64 on the finite-difference test's data.
# Measured on B200 over 40 steps: 1.4e-3 (relative L2), with FP64's
# cotangent or with its own.  The scheme is differentiable almost everywhere:
# near extrema the limiter's choice sits close to a switch, and where the
# FP32 and FP64 forward states fall on different sides the two adjoints take
# different branches there.
FP32_ADJOINT_REL_L2 = 5e-3
FP32_GRADIENT_REL_L2 = 5e-3


def test_fp32_gradient_agrees_with_fp64(pkg):
    n, steps = 128, 40
    U, w, h, hh = vortex_case(pkg, n, seed=3)
    Ut, _, _, _ = vortex_case(pkg, n, seed=11)
    dt = fixed_dt(pkg, U, hh)
    target = forward(pkg, Ut, w, h, dt, steps)[..., 0]
    g64, cot64 = gradient(pkg, U, w, h, dt, steps, target, pkg.FP64)
    g32, _ = gradient(pkg, U, w, h, dt, steps, target, pkg.FP32, cot=cot64)
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    print("fp32 adjoint of the fp64 cotangent: rel L2", rel)
    assert rel <= FP32_ADJOINT_REL_L2, rel
    g32own, _ = gradient(pkg, U, w, h, dt, steps, target, pkg.FP32)
    rel = np.linalg.norm(g32own - g64) / np.linalg.norm(g64)
    print("fp32 gradient with its own cotangent: rel L2", rel)
    assert rel <= FP32_GRADIENT_REL_L2, rel


# Measured on B200: 1.2e-7 to 8e-7 (relative L2) on six presets, 1.4e-4 on
# the seventh's data, where a cell's limiter choice flips between the FP32
# and FP64 forward states.
def test_fp32_vjp_of_one_step_every_preset_agrees_with_fp64(pkg, oracle):
    for strategy in range(7):
        n = 48
        U = oracle.ghost(pkg.scenarios.seeded_four_quadrant(n, 40, 90 + strategy), strategy)
        dt = fixed_dt(pkg, U, 1.0 / n) * 0.5
        wv = np.random.default_rng(strategy).standard_normal(U.shape)
        out = []
        for prec in (pkg.FP64, pkg.FP32):
            hd = pkg.Handle(n, 40)
            hd.configure(1.0, 40 / n, 1e9, 0.45, 1.9, 1.4, strategy, prec)
            hd.set_fixed_dt(dt)
            hd.set_state(U)
            hd.forward(1, 1)
            out.append(hd.vjp(wv))
            hd.close()
        rel = np.linalg.norm(out[1] - out[0]) / np.linalg.norm(out[0])
        print("preset", strategy, "fp32 vjp rel L2 vs fp64", rel)
        assert rel <= 1e-3, (strategy, rel)


def diff_handle(pkg, U, w, h, dt, precision):
    ny, nx = U.shape[:2]
    hd = pkg.Handle(nx, ny)
    hd.configure(w, h, 1e9, 0.45, 1.9, 1.4, 5, precision)
    hd.set_fixed_dt(dt)
    hd.set_state(U)
    return hd


# The ghost ring's transpose accumulates with atomics, so two VJPs of the
# same tape may differ in the last bits: relative L2 bounds, not equality.
@pytest.mark.parametrize("precision,tol", [("FP64", 1e-12), ("FP32", 1e-5)])
def test_full_tape_matches_checkpoints(pkg, precision, tol):
    n, steps = 96, 25
    U, w, h, hh = vortex_case(pkg, n)
    dt = fixed_dt(pkg, U, hh)
    wv = np.random.default_rng(5).standard_normal(U.shape)
    prec = getattr(pkg, precision)
    out = {}
    for ck in (5, pkg.FULL_TAPE):
        hd = diff_handle(pkg, U, w, h, dt, prec)
        hd.forward(steps, ck)
        final = hd.get_state(4)
        g = hd.vjp(wv)
        assert np.array_equal(hd.get_state(4), final)  # the reverse leaves the final state in place
        out[ck] = (final, g, hd.time_stages_count())
        if ck == pkg.FULL_TAPE:
            g2 = hd.vjp(2.0 * wv)  # the tape serves another cotangent without a new forward
            rel = np.linalg.norm(g2 - 2.0 * g) / np.linalg.norm(2.0 * g)
            assert rel <= tol, rel
        hd.close()
    (f5, g5, n5), (ft, gt, nt) = out[5], out[pkg.FULL_TAPE]
    assert n5 == nt == steps
    print(precision, "final state bit-identical:", np.array_equal(f5, ft))
    assert np.allclose(ft, f5, rtol=tol, atol=0)
    rel = np.linalg.norm(gt - g5) / np.linalg.norm(g5)
    print(precision, "full tape vs checkpoints: cotangent rel L2", rel)
    assert rel <= tol, rel


def test_full_tape_is_discarded_by_a_parameter_change(pkg):
    U, w, h, hh = vortex_case(pkg, 64)
    dt = fixed_dt(pkg, U, hh)
    hd = diff_handle(pkg, U, w, h, dt, pkg.FP64)
    hd.forward(6, pkg.FULL_TAPE)
    wv = np.ones_like(U)
    hd.vjp(wv)
    hd.configure(w, h, 1e9, 0.45, 1.8, 1.4, 5, pkg.FP64)  # alpha changed: the tape is stale
    with pytest.raises(pkg.FVM2DError, match="call it first"):
        hd.vjp(wv)
    with pytest.raises(pkg.FVM2DError, match="use checkpoints"):
        hd.forward(10**8, pkg.FULL_TAPE)  # rejected before any allocation
    hd.forward(6, pkg.FULL_TAPE)
    assert np.isfinite(hd.vjp(wv)).all()
    hd.close()
