"""Row-slab decomposition of one problem across processes (2d_fvm_cuda_b200/slab.py),
tested on CPU: gloo ranks whose slabs are stepped by the oracle-backed
stand-in of tests/slab_ranks.py, on every ghost preset.  The gathered result
must equal the oracle's single-array run bit for bit: same steps, same time,
same cells."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import slab_ranks


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_plan_covers_the_rows_once(pkg):
    sl = pkg.slab
    for ny, world in [(40, 2), (41, 3), (1024, 8), (16, 4)]:
        slabs = sl.plan_slabs(ny, world)
        assert slabs[0][0] == 0 and slabs[-1][1] == ny
        assert all(a[1] == b[0] for a, b in zip(slabs, slabs[1:]))
        assert all(hi - lo >= sl.MIN_ROWS for lo, hi in slabs)
    with pytest.raises(ValueError):
        sl.plan_slabs(15, 4)


def test_halo_messages_fill_every_halo_row(pkg):
    sl = pkg.slab
    for ny, world, strategy in [(40, 2, 0), (41, 3, 5), (64, 4, 6), (30, 2, 5)]:
        slabs = sl.plan_slabs(ny, world)
        got = {r: set() for r in range(world)}
        for src, dst, g_send, g_recv in sl.halo_messages(ny, world, strategy):
            lo, hi = slabs[src]
            assert lo <= g_send and g_send + sl.HALO <= hi  # sent rows are the sender's own
            l_lo, l_hi = sl.local_rows(ny, world, dst)
            assert l_lo <= g_recv and g_recv + sl.HALO <= l_hi
            got[dst] |= {g_recv, g_recv + 1}
        for r in range(world):
            l_lo, l_hi = sl.local_rows(ny, world, r)
            lo, hi = slabs[r]
            want = set(range(l_lo, lo)) | set(range(hi, l_hi))
            if strategy == 5 and world > 1:
                want |= {0, 1} if r == 0 else set()
                want |= {ny - 2, ny - 1} if r == world - 1 else set()
            assert got[r] == want, (ny, world, strategy, r)


CASES = [
    dict(world=2, nx=64, ny=57, seed=3, strategy=0, width=1.0, height=1.1, t_end=0.05, steps=12),
    dict(world=3, nx=33, ny=46, seed=4, strategy=5, width=1.0, height=1.0, t_end=0.05, steps=12),
    dict(world=2, nx=40, ny=30, seed=5, strategy=6, width=1.2, height=1.0, t_end=0.05, steps=12),
    # presets whose ghost rules read global row numbers (double-Mach shock
    # position, jet inflow rows)
    dict(world=3, nx=48, ny=40, seed=6, strategy=4, width=1.0, height=1.0, t_end=0.02, steps=10),
    dict(world=2, nx=48, ny=42, seed=7, strategy=1, width=1.0, height=1.0, t_end=0.02, steps=10),
    dict(world=3, nx=40, ny=50, seed=8, strategy=2, width=1.0, height=1.0, t_end=0.001, steps=10),
    dict(world=2, nx=40, ny=44, seed=9, strategy=3, width=1.0, height=1.0, t_end=0.001, steps=10),
    # the state given as a function of the rows, and a restart from it
    dict(world=3, nx=36, ny=47, seed=11, strategy=0, width=1.0, height=1.0, t_end=0.05, steps=9, rows_fn=True),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"world{c['world']}-strategy{c['strategy']}"
                         + ("-rows_fn" if c.get("rows_fn") else ""))
def test_slab_run_equals_single_array_run(oracle, case, tmp_path):
    out = str(tmp_path / "gathered.npz")
    mp.spawn(slab_ranks.cpu_worker, args=(case["world"], free_port(), case, out), nprocs=case["world"], join=True)
    z = np.load(out)
    G, t, steps = z["G"], float(z["t"]), int(z["steps"])
    U = slab_ranks.initial_state(case["nx"], case["ny"], case["seed"], case["strategy"])
    R, rsteps, rt = oracle.solve(U, max_steps=case["steps"], width=case["width"], height=case["height"], cfl=0.45,
                                 alpha=1.9, gamma=1.4, t_end=case["t_end"], strategy=case["strategy"])
    assert (steps, t) == (rsteps, rt)
    assert np.array_equal(G, R, equal_nan=True)
    # the ranks' conserved totals (each its own rows) add up to the whole
    # interior's, which the one-array run gives
    V = R[2:-2, 2:-2]
    r, p, u, v = V[..., 0], V[..., 1], V[..., 2], V[..., 3]
    area = (case["width"] / case["nx"]) * (case["height"] / case["ny"])
    parts = (r, r * u, r * v, p / 0.4 + 0.5 * r * (u * u + v * v))
    want = np.array([np.sum(x) for x in parts]) * area
    scale = np.array([np.sum(np.abs(x)) for x in parts]) * area
    assert np.all(np.abs(z["totals"] - want) <= 1e-13 * scale), (z["totals"], want)
