"""Per-rank worker of the ensemble tests: gloo ranks split a list of small
problems with 2d_fvm_cuda_b200.ensemble and solve their share with the
oracle (the checker, standing in for the GPU batch on CPU)."""
import datetime
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

SIZES = [(48, 32), (64, 64), (37, 29), (96, 48), (32, 80), (40, 40), (16, 16), (72, 24), (24, 72)]


def problems():
    """Mixed sizes, all seven presets, different end times and parameters."""
    pkg = importlib.import_module("2d_fvm_cuda_b200")
    from oracle import Oracle

    orc = Oracle(threads=1)
    out = []
    for k, (nx, ny) in enumerate(SIZES):
        s = k % 7
        U = pkg.scenarios.seeded_four_quadrant(nx, ny, 700 + k)
        if s in (5, 6):
            U = orc.ghost(U, s)
        out.append((U, dict(width=1.0 + 0.1 * k, height=1.0, t_end=0.004 + 0.003 * k, cfl=0.45,
                            alpha=1.5 + 0.05 * k, gamma=1.4, strategy=s)))
    return out


def oracle_solve(share, precision, rank=0):
    """A rank's share solved one problem at a time by the oracle; each result
    carries the rank that computed it."""
    from oracle import Oracle

    orc = Oracle(threads=1)
    out = []
    for U, kw in share:
        V, steps, t = orc.solve(U, **kw)
        out.append((V, t, steps, rank))
    return out


def cpu_worker(rank, world, port, out_path):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        pkg = importlib.import_module("2d_fvm_cuda_b200")
        E = pkg.ensemble.EnsembleSolver(problems(), precision=1,
                                        solve=lambda share, prec: oracle_solve(share, prec, rank))
        E.solve()
        got = E.gather()
        if rank == 0:  # through a file: a pipe would block on results above its 64 KB buffer
            np.savez(out_path, **{f"U{i}": g[0] for i, g in enumerate(got)},
                     t=np.array([g[1] for g in got]), steps=np.array([g[2] for g in got]),
                     rank=np.array([g[3] for g in got]), plan=np.array([r for i in range(len(got))
                                                                        for r, s in enumerate(E.plan) if i in s]))
    finally:
        dist.destroy_process_group()
