"""Batched form: many independent problems of different sizes in one set of
launches per step.  Per problem, the contraction-free build (FP64_STRICT)
must give exactly what a solve of that problem alone gives (same steps, same
final time, same bits) and what the oracle gives.  The builds with FMA
contraction inline the same arithmetic into two different kernels, where the
compiler may contract it differently, so they must agree with the single
solve to rounding: the parity tolerance (relative L1 1e-10 per field) for
FP64, and for FP32 its own rounding level."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = [(48, 32), (64, 64), (37, 29), (96, 48), (32, 80), (128, 128), (16, 16), (200, 72)]
STRATEGIES = [0, 1, 2, 3, 4, 5, 6, 0]


def problems(pkg, oracle):
    out = []
    for k, (nx, ny) in enumerate(SIZES):
        U = pkg.scenarios.seeded_four_quadrant(nx, ny, 500 + k)
        s = STRATEGIES[k]
        if s in (5, 6):
            U = oracle.ghost(U, s)
        kw = dict(width=1.0 + 0.1 * k, height=1.0, t_end=0.004 + 0.002 * k, cfl=0.45, alpha=1.5 + 0.05 * k,
                  gamma=1.4, strategy=s)
        out.append((U, kw))
    return out


def single(pkg, U, kw, precision):
    ny, nx = U.shape[:2]
    h = pkg.Handle(nx, ny)
    h.configure(kw["width"], kw["height"], kw["t_end"], kw["cfl"], kw["alpha"], kw["gamma"], kw["strategy"],
                precision)
    h.set_state(U)
    h.solve()
    t, steps, _ = h.time()
    V = h.get_state(4)
    h.close()
    return V, steps, t


def batch_solve(pkg, probs, precision, tune=False):
    b = pkg.Batch([(U.shape[1], U.shape[0]) for U, _ in probs])
    b.set_precision(precision)
    for p, (U, kw) in enumerate(probs):
        b.set_problem(p, **kw)
        b.set_state(p, U)
    if tune:
        b.autotune(2)
    b.solve()
    out = [(b.get_state(p), *b.time(p)[::-1]) for p in range(len(probs))]
    stats = b.run_stats()
    b.close()
    return out, stats


REL_L1 = {0: 1e-10, 3: 2e-4}  # per field, batch vs single, contracting builds (FP32: measured 5e-5 on the jet)


def rel_l1(A, B):
    return max(np.nansum(np.abs(A[..., f] - B[..., f])) / np.nansum(np.abs(B[..., f])) for f in range(4))


def agree(precision, G, V, gsteps, steps):
    if precision == 1:
        return gsteps == steps and np.array_equal(G, V, equal_nan=True)
    if precision == 3:
        return abs(gsteps - steps) <= 1 and rel_l1(G, V) <= REL_L1[3]
    return gsteps == steps and rel_l1(G, V) <= REL_L1[0]


@pytest.mark.parametrize("precision", [1, 0, 3])
def test_batch_agrees_with_single_solves(pkg, oracle, precision):
    probs = problems(pkg, oracle)
    got, stats = batch_solve(pkg, probs, precision)
    cells = 0
    for p, (U, kw) in enumerate(probs):
        V, steps, t = single(pkg, U, kw, precision)
        G, gsteps, gt = got[p]
        assert gt == pytest.approx(kw["t_end"], abs=1e-15) and t == pytest.approx(kw["t_end"], abs=1e-15)
        assert agree(precision, G, V, gsteps, steps), (p, gsteps, steps, rel_l1(G, V))
        cells += U.shape[0] * U.shape[1] * gsteps
    assert stats[2] == cells


@pytest.mark.parametrize("precision", [1, 0])
def test_batch_after_autotune_agrees_with_single_solves(pkg, oracle, precision):
    probs = problems(pkg, oracle)
    got, _ = batch_solve(pkg, probs, precision, tune=True)
    for p, (U, kw) in enumerate(probs):
        V, steps, t = single(pkg, U, kw, precision)
        assert agree(precision, got[p][0], V, got[p][1], steps), p


def test_strict_batch_equals_oracle(pkg, oracle):
    probs = problems(pkg, oracle)[:4]
    got, _ = batch_solve(pkg, probs, 1)
    for p, (U, kw) in enumerate(probs):
        O, steps, t = oracle.solve(U, **{k: kw[k] for k in ("width", "height", "cfl", "alpha", "gamma", "t_end",
                                                              "strategy")})
        assert got[p][1:] == (steps, t)
        assert np.array_equal(got[p][0], O, equal_nan=True)


def test_ensemble_without_a_process_group_is_one_batch(pkg, oracle):
    """2d_fvm_cuda_b200.ensemble on a single process: its default share
    solver runs the whole list as one batch, bit for bit the batch above."""
    probs = problems(pkg, oracle)
    want, _ = batch_solve(pkg, probs, 1)
    E = pkg.ensemble.EnsembleSolver(probs, precision=1)
    assert E.solve() == len(probs)
    for (G, steps, t), (V, tt, ss) in zip(want, E.gather()):
        assert (ss, tt) == (steps, t)
        assert np.array_equal(V, G, equal_nan=True)
