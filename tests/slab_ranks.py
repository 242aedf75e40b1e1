"""Per-rank workers of the slab tests, and the CPU stand-in for a slab's GPU
solver used by the CPU ones.  The stand-in steps its rows with the oracle's
sweeps and ghost fill (the oracle is the checker here) and follows the GPU
solver's row-frame rules: the row spacing is the whole problem's, the ghost
presets see global row numbers and fill only the problem's own edges, and
after a step the halo rows it does not own are left out of its wave-speed
maximum."""
import datetime
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for _p in (ROOT, os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)


class OracleSlab:
    def __init__(self, orc, nx, ny):
        self.orc, self.nx, self.ny = orc, nx, ny
        self.t, self.fresh = 0.0, True

    def configure(self, width, height, t_end, cfl, alpha, gamma, strategy, precision):
        self.width, self.height, self.alpha, self.gamma, self.strategy = width, height, alpha, gamma, strategy

    def set_row_frame(self, row0, ny_global, fill_top, fill_bottom):
        self.row0, self.ny_global, self.fill_top, self.fill_bottom = row0, ny_global, fill_top, fill_bottom

    def set_state(self, U):
        self.U = np.ascontiguousarray(U[..., :4], dtype=np.float64).copy()
        self.fresh = True

    def wave_speed_max(self):
        if self.fresh:
            return self.orc.max_speed(self.U, self.gamma)
        a = 0 if self.fill_top else 2
        b = self.ny if self.fill_bottom else self.ny - 2
        return self.orc.max_speed(self.U[a:b], self.gamma)

    def sweep_y(self, U, dt, **kw):
        """The oracle's y-sweep with the problem's row spacing height / ny_global:
        the slab is padded below to ny_global rows by copies of its last row.
        Padding reaches only the slab's last two rows, which are halo or ghost
        rows that the exchange or the ghost fill replaces."""
        P = np.concatenate([U, np.repeat(U[-1:], self.ny_global - self.ny, axis=0)])
        return self.orc.sweep_y(P, self.height, dt, **kw)[:self.ny]

    def advance_dt(self, dt):
        o, kw = self.orc, dict(alpha=self.alpha, gamma=self.gamma)
        A = self.sweep_y(o.sweep_x(self.U, self.width, dt, **kw), dt, **kw)
        B = o.sweep_x(self.sweep_y(self.U, dt, **kw), self.width, dt, **kw)
        V = (A + B) * 0.5
        self.t = self.t + dt
        self.U = self.ghost(V)
        self.fresh = False

    def ghost(self, V):
        """The oracle's ghost fill of the whole problem, on the slab placed at
        its global rows (the other rows are zeros: the presets only copy
        them, and the slab keeps none of them), then the slab's rows that the
        frame fills: its ring columns on every row it owns and, on the
        problem's own edges, its two ring rows; halo rows stay as the
        exchange left them."""
        G = np.zeros((self.ny_global, self.nx, 4))
        G[self.row0:self.row0 + self.ny] = V
        G = self.orc.ghost(G, self.strategy, t=self.t, width=self.width, height=self.height)
        a = 0 if self.fill_top else 2
        b = self.ny if self.fill_bottom else self.ny - 2
        V = V.copy()
        V[a:b] = G[self.row0 + a:self.row0 + b]
        return V

    def conserved_totals(self):
        """The library's interior totals (rows and columns 2 .. n-3 of the
        slab's array, the problem's row spacing), summed exactly."""
        import math
        V = self.U[2:-2, 2:-2]
        r, p, u, v = V[..., 0], V[..., 1], V[..., 2], V[..., 3]
        area = (self.width / self.nx) * (self.height / self.ny_global)
        parts = (r, r * u, r * v, p / (self.gamma - 1) + 0.5 * r * (u * u + v * v))
        return np.array([math.fsum(x.ravel()) for x in parts]) * area

    def get_rows(self, j0, nrows, out=None):
        R = np.ascontiguousarray(np.moveaxis(self.U[j0:j0 + nrows], -1, 0))
        if out is None:
            return R
        out[...] = R
        return out

    def set_rows(self, j0, rows):
        rows = np.asarray(rows).reshape(4, -1, self.nx)
        self.U[j0:j0 + rows.shape[1]] = np.moveaxis(rows, 0, -1)

    def close(self):
        pass


def initial_state(nx, ny, seed, strategy):
    pkg = importlib.import_module("2d_fvm_cuda_b200")
    U = pkg.scenarios.seeded_four_quadrant(nx, ny, seed)
    if strategy == 5:  # a state whose ghost rows already wrap
        from oracle import Oracle
        U = Oracle(threads=1).ghost(U, 5)
    return U


def _init(rank, world, port):
    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    return dist


def cpu_worker(rank, world, port, case, out_path):
    dist = _init(rank, world, port)
    try:
        pkg = importlib.import_module("2d_fvm_cuda_b200")
        from oracle import Oracle

        orc = Oracle(threads=1)
        U = initial_state(case["nx"], case["ny"], case["seed"], case["strategy"])
        kw = dict(width=case["width"], height=case["height"], t_end=case["t_end"], cfl=0.45, alpha=1.9, gamma=1.4,
                  strategy=case["strategy"], make_local=lambda nx, rows: OracleSlab(orc, nx, rows))
        if case.get("rows_fn"):
            # the state given as a function of the global rows; a few steps,
            # then this rank's rows loaded again and the run restarted
            S = pkg.slab.SlabSolver(lambda lo, hi: U[lo:hi], shape=U.shape[:2], **kw)
            S.advance(3)
            S.set_local_state(U[S.l_lo:S.l_hi])
        else:
            S = pkg.slab.SlabSolver(U, **kw)
        S.advance(case["steps"])
        T = S.conserved_totals()
        G = S.gather()
        if rank == 0:  # through a file: a pipe would block on results above its 64 KB buffer
            np.savez(out_path, G=G, t=S.t, steps=S.steps, totals=T)
    finally:
        dist.destroy_process_group()


def gpu_worker(rank, world, port, case, out_path):
    """A rank with the real GPU solver (libfvm2d); ranks share one GPU and
    exchange rows through host memory (gloo).  No kernel waits on another
    rank: the exchange happens between steps, on the host."""
    dist = _init(rank, world, port)
    try:
        pkg = importlib.import_module("2d_fvm_cuda_b200")
        U = pkg.scenarios.seeded_four_quadrant(case["nx"], case["ny"], case["seed"])
        S = pkg.slab.SlabSolver(U, width=case["width"], height=case["height"], t_end=case["t_end"], cfl=0.45,
                                alpha=1.9, gamma=1.4, strategy=case["strategy"], precision=case["precision"])
        S.solve()
        G = S.gather()
        S.close()
        if rank == 0:  # through a file: a pipe would block on results above its 64 KB buffer
            np.savez(out_path, G=G, t=S.t, steps=S.steps)
    finally:
        dist.destroy_process_group()


def nccl_worker(rank, world, port, case, out_path):
    """One rank per GPU over NCCL: the steps are enqueued on the device (halo
    rows packed, exchanged and unpacked on the handle's stream, the wave-speed
    max reduced on the device and the step planned from it), no host round
    trip per step.  With one GPU the group has one rank."""
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(rank)
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", rank))
    try:
        pkg = importlib.import_module("2d_fvm_cuda_b200")
        U = pkg.scenarios.seeded_four_quadrant(case["nx"], case["ny"], case["seed"])
        S = pkg.slab.SlabSolver(lambda lo, hi: U[lo:hi], shape=U.shape[:2], width=case["width"],
                                height=case["height"], t_end=case["t_end"], cfl=0.45, alpha=1.9, gamma=1.4,
                                strategy=case["strategy"], precision=case["precision"])
        assert S.on_device
        k = S.advance(case["first"])  # a fixed number of steps, then the rest of the run in groups
        S.solve(check_every=5)
        G = S.gather()
        S.close()
        if rank == 0:
            np.savez(out_path, G=G, t=S.t, steps=S.steps, first=k)
    finally:
        dist.destroy_process_group()
