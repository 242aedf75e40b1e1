"""Independent problems dealt out whole across processes
(2d_fvm_cuda_b200/ensemble.py), tested on CPU: the plan gives every problem
to exactly one rank with balanced estimated work, and gloo ranks that solve
their share with the oracle gather exactly what solving every problem alone
gives, each problem computed by the rank the plan names."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import ensemble_ranks


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_plan_gives_each_problem_to_one_rank_with_balanced_work(pkg):
    en = pkg.ensemble
    rng = np.random.default_rng(0)
    for n, world in [(1, 1), (5, 8), (100, 3), (1024, 8), (37, 4)]:
        costs = rng.lognormal(0.0, 1.5, n)
        plan = en.plan_shards(costs, world)
        assert len(plan) == world
        assert sorted(i for s in plan for i in s) == list(range(n))
        assert all(s == sorted(s) for s in plan)
        loads = [costs[s].sum() if s else 0.0 for s in plan]
        # longest processing time first: no rank above the mean by more than
        # one problem's cost
        assert max(loads) <= costs.sum() / world + costs.max() + 1e-9
        assert plan == en.plan_shards(list(costs), world)  # the same on every rank
    with pytest.raises(ValueError):
        en.plan_shards([1.0], 0)


def test_cost_grows_with_size_and_end_time(pkg):
    c = pkg.ensemble.estimated_cost
    assert c(64, 64, t_end=0.2, cfl=0.45) < c(128, 128, t_end=0.2, cfl=0.45) < c(128, 128, t_end=0.4, cfl=0.45)
    assert c(64, 64, t_end=0.0) == 64 * 64  # at least one step


def test_one_process_solves_everything(pkg, oracle):
    probs = ensemble_ranks.problems()[:4]
    E = pkg.ensemble.EnsembleSolver(probs, precision=1, solve=ensemble_ranks.oracle_solve)
    assert (E.rank, E.world, E.mine) == (0, 1, [0, 1, 2, 3])
    assert E.solve() == 4
    for (U, kw), (V, t, steps, _) in zip(probs, E.gather()):
        R, rsteps, rt = oracle.solve(U, **kw)
        assert (steps, t) == (rsteps, rt) and np.array_equal(V, R, equal_nan=True)


@pytest.mark.parametrize("world", [2, 3])
def test_ranks_gather_what_single_solves_give(pkg, oracle, world, tmp_path):
    out = str(tmp_path / "gathered.npz")
    mp.spawn(ensemble_ranks.cpu_worker, args=(world, free_port(), out), nprocs=world, join=True)
    z = np.load(out)
    probs = ensemble_ranks.problems()
    assert sorted(set(z["rank"].tolist())) == list(range(world))  # every rank had work
    assert np.array_equal(z["rank"], z["plan"])  # each problem solved where the plan put it
    for i, (U, kw) in enumerate(probs):
        R, rsteps, rt = oracle.solve(U, **kw)
        assert (int(z["steps"][i]), float(z["t"][i])) == (rsteps, rt), i
        assert np.array_equal(z[f"U{i}"], R, equal_nan=True), i
