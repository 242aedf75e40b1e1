"""One problem split by rows across processes, one GPU each (row slabs).

The reference is single-device (src/wrappers.cuh:154-306).  Here its loop is
spread over the ranks of a ``torch.distributed`` process group:

* The array's rows are cut into contiguous slabs, one per rank.  A rank's
  solver holds its slab plus two halo rows on every inner edge.
* A step updates row j from U^n on rows j-2 .. j+2 in both split orders
  (Y(X(U)) reads X(U) on rows j±2, which the rank computes itself from its
  halo; X(Y(U)) reads Y(U) on row j), so before every step each rank sends
  its first and last two rows to its neighbours and receives their two rows
  into its halo.  With the periodic preset the first and last slabs also swap
  the wrapped rows (0, 1 <- ny-4, ny-3 and ny-2, ny-1 <- 2, 3).
* The step size is the reference's rule (src/wrappers.cuh:196-207) applied to
  the wave-speed maximum reduced over all ranks: one 8-byte all-reduce.
* The presets fill only the problem's own edges and see global row numbers
  (the solver's row frame); halo rows are left out of each rank's maximum.

Every rank computes exactly the cells a single device would, with the same
arithmetic and the same dt, so the gathered result equals a single-device
run bit for bit.  With the NCCL backend the halo rows travel between device
buffers; with any other backend through host memory.

With NCCL and the library's solver handle the steps never wait on the host:
the rows are packed and unpacked, the halos exchanged, the wave-speed maximum
reduced (8 bytes, on the device) and the next step planned from it by a
kernel, all enqueued in order on the handle's own CUDA stream (NCCL runs on
a torch stream wrapping it).  The host reads the time back only when asked
(``sync``) or every few steps of ``solve``.  Other backends, or a stand-in
solver, take the host-driven path (``step``): the maximum read back to the
host and the dt computed there.
"""
from __future__ import annotations

import numpy as np

OUTFLOW, REFLECTIVE, JET, JET800, DOUBLE_MACH, PERIODIC, REFLECTIVE_TB = range(7)
HALO = 2
MIN_ROWS = 4  # rows a slab must own: its neighbours read two from each end


def plan_slabs(ny: int, world: int) -> list[tuple[int, int]]:
    """Owned global rows [lo, hi) of each rank: ny rows split evenly."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    base, extra = divmod(ny, world)
    if base < MIN_ROWS:
        raise ValueError(f"{ny} rows cannot give each of {world} ranks {MIN_ROWS} rows")
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def local_rows(ny: int, world: int, rank: int) -> tuple[int, int]:
    """Global rows [l_lo, l_hi) a rank's solver holds: its slab plus halos."""
    lo, hi = plan_slabs(ny, world)[rank]
    return (lo - HALO if rank > 0 else 0), (hi + HALO if rank < world - 1 else ny)


def halo_messages(ny: int, world: int, strategy: int) -> list[tuple[int, int, int, int]]:
    """Every row transfer of one exchange as (src rank, dst rank, first global
    row sent, first global row received), two rows each, in one fixed order
    that all ranks follow."""
    slabs = plan_slabs(ny, world)
    msgs = []
    for r in range(world - 1):
        lo_n, hi_r = slabs[r + 1][0], slabs[r][1]
        msgs.append((r, r + 1, hi_r - HALO, hi_r - HALO))  # last rows of r -> top halo of r+1
        msgs.append((r + 1, r, lo_n, lo_n))                 # first rows of r+1 -> bottom halo of r
    if strategy == PERIODIC and world > 1:
        msgs.append((world - 1, 0, ny - 4, 0))  # rows ny-4, ny-3 -> ghost rows 0, 1
        msgs.append((0, world - 1, 2, ny - 2))  # rows 2, 3 -> ghost rows ny-2, ny-1
    return msgs


def row_frame(ny: int, world: int, rank: int, strategy: int) -> tuple[int, int, bool, bool]:
    """(row0, ny_global, fill_top, fill_bottom) of a rank's solver."""
    l_lo, _ = local_rows(ny, world, rank)
    wrap = strategy == PERIODIC and world > 1
    return l_lo, ny, rank == 0 and not wrap, rank == world - 1 and not wrap


class SlabSolver:
    """This rank's part of a problem of ny x nx cells (ghost layers included).

    ``U`` is the whole initial state, shape (ny, nx, 4|5), on every rank (each
    keeps its rows), or a function ``U(lo, hi)`` returning global rows
    [lo, hi) of it, in which case ``shape`` = (ny, nx) gives the problem's
    size.  ``make_local(nx, rows)`` builds the rank's solver (a ``Handle`` by
    default); ``group`` is the process group (default: WORLD).
    """

    def __init__(self, U, width=1.0, height=1.0, t_end=0.0, cfl=0.5, alpha=1.9, gamma=1.4, strategy=OUTFLOW,
                 precision=0, group=None, make_local=None, shape=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        if callable(U):
            if shape is None:
                raise ValueError("shape=(ny, nx) is required when U is a function of the rows")
            self.ny, self.nx = int(shape[0]), int(shape[1])
            rows_of = U
        else:
            U = np.asarray(U, dtype=np.float64)
            self.ny, self.nx = U.shape[:2]
            rows_of = lambda lo, hi: U[lo:hi]  # noqa: E731
        self.strategy = int(strategy)
        self.l_lo, self.l_hi = local_rows(self.ny, self.world, self.rank)
        self.lo, self.hi = plan_slabs(self.ny, self.world)[self.rank]
        self.rows = self.l_hi - self.l_lo
        hx, hy = width / self.nx, height / self.ny
        self.hmin = hy if hy < hx else hx
        self.t_end, self.cfl = float(t_end), float(cfl)
        self.t, self.steps, self.done = 0.0, 0, False
        self.fresh = True  # every halo holds true rows (the initial scatter, or an exchange after a step)
        if make_local is None:
            from ._lib import Handle as make_local
        self.local = make_local(self.nx, self.rows)
        # the whole problem's height: with the row frame the solver keeps the row spacing height / ny
        self.local.configure(width, height, t_end, cfl, alpha, gamma, self.strategy, precision)
        row0, gny, top, bottom = row_frame(self.ny, self.world, self.rank, self.strategy)
        self.local.set_row_frame(row0, gny, top, bottom)
        self.local.set_state(np.ascontiguousarray(rows_of(self.l_lo, self.l_hi), dtype=np.float64))
        self.device = dist.get_backend(group) == "nccl"
        self.msgs = halo_messages(self.ny, self.world, self.strategy)
        self._bufs = [self._buffer() for _ in self.msgs]
        # steps enqueued on the device, no host round trip (NCCL + the library's handle)
        self.on_device = self.device and hasattr(self.local, "slab_step")
        if self.on_device:
            import torch

            self._stream = torch.cuda.ExternalStream(self.local.stream_ptr())
            self._smax_local = torch.zeros(1, dtype=torch.float64, device="cuda")
            self._smax_all = torch.zeros(1, dtype=torch.float64, device="cuda")
            self._begun = False

    # ---- buffers -------------------------------------------------------------
    def _buffer(self, rows=HALO):
        import torch

        if self.device:
            return torch.empty((4, rows, self.nx), dtype=torch.float64, device="cuda")
        return torch.empty((4, rows, self.nx), dtype=torch.float64)

    def _rows_out(self, g0, buf):
        j0 = g0 - self.l_lo
        if self.device:
            self.local.get_rows_ptr(j0, buf.shape[1], buf.data_ptr())
        else:
            self.local.get_rows(j0, buf.shape[1], out=buf.numpy())

    def _rows_in(self, g0, buf):
        j0 = g0 - self.l_lo
        if self.device:
            import torch

            torch.cuda.current_stream().synchronize()  # the transfer ran on torch's stream
            self.local.set_rows_ptr(j0, buf.shape[1], buf.data_ptr())
        else:
            self.local.set_rows(j0, buf.numpy())

    def _global(self, r: int) -> int:
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def set_local_state(self, R) -> None:
        """Replaces this rank's rows (its slab and halo rows: global rows
        l_lo .. l_hi-1, shape (l_hi - l_lo, nx, 4|5), host or pinned memory)
        and restarts the run at t = 0."""
        self.local.set_state(R)
        self.t, self.steps, self.done, self.fresh = 0.0, 0, False, True
        if self.on_device:
            self._begun = False

    # ---- one step ------------------------------------------------------------
    def exchange(self) -> None:
        """Fills this rank's halo rows from its neighbours."""
        if not self.msgs:
            return
        dist = self.dist
        ops, recvs = [], []
        for k, (src, dst, g_send, g_recv) in enumerate(self.msgs):
            buf = self._bufs[k]
            if src == self.rank:
                self._rows_out(g_send, buf)
                ops.append(dist.P2POp(dist.isend, buf, self._global(dst), self.group, k))
            elif dst == self.rank:
                ops.append(dist.P2POp(dist.irecv, buf, self._global(src), self.group, k))
                recvs.append((g_recv, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for g_recv, buf in recvs:
            self._rows_in(g_recv, buf)

    def global_wave_speed_max(self) -> float:
        import torch

        v = torch.tensor([self.local.wave_speed_max()], dtype=torch.float64,
                         device="cuda" if self.device else "cpu")
        self.dist.all_reduce(v, op=self.dist.ReduceOp.MAX, group=self.group)
        return float(v.item())

    # ---- steps enqueued on the device (NCCL) --------------------------------------
    def _exchange_on_stream(self) -> None:
        """The halo exchange, enqueued on the handle's stream (the caller has
        made it torch's current stream)."""
        dist = self.dist
        ops, recvs = [], []
        for k, (src, dst, g_send, g_recv) in enumerate(self.msgs):
            buf = self._bufs[k]
            if src == self.rank:
                self.local.get_rows_async(g_send - self.l_lo, HALO, buf.data_ptr())
                ops.append(dist.P2POp(dist.isend, buf, self._global(dst), self.group, k))
            elif dst == self.rank:
                ops.append(dist.P2POp(dist.irecv, buf, self._global(src), self.group, k))
                recvs.append((g_recv, buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()  # NCCL: the stream waits, the host does not
        for g_recv, buf in recvs:
            self.local.set_rows_async(g_recv - self.l_lo, HALO, buf.data_ptr())

    def enqueue_steps(self, n: int) -> None:
        """Enqueues n steps of the whole problem (NCCL path); returns without
        waiting.  Steps after the loop has ended do nothing."""
        import torch

        with torch.cuda.stream(self._stream):
            for _ in range(n):
                if not self._begun:
                    self.local.slab_begin(self._smax_local.data_ptr())
                    self._begun = True
                elif not self.fresh:
                    self._exchange_on_stream()
                self._smax_all.copy_(self._smax_local)
                self.dist.all_reduce(self._smax_all, op=self.dist.ReduceOp.MAX, group=self.group)
                self.local.slab_step(self._smax_all.data_ptr(), self._smax_local.data_ptr())
                self.fresh = False

    def sync(self) -> tuple[float, int, bool]:
        """Waits for the enqueued steps; (t, steps, done).  Every rank reaches
        the same values (the same dt everywhere)."""
        self.t, self.steps, self.done = self.local.slab_sync()
        return self.t, self.steps, self.done

    def step(self) -> bool:
        """One step of the whole problem; False once the loop has ended."""
        if self.on_device:
            if self.done:
                return False
            before = self.steps
            self.enqueue_steps(1)
            return self.sync()[1] > before
        if self.done:
            return False
        if not self.fresh:
            self.exchange()
        smax = self.global_wave_speed_max()
        # src/wrappers.cuh:196-207, as the device plans it
        if not (self.t < self.t_end):
            self.done = True
            return False
        a, b = self.cfl * self.hmin / smax, self.t_end - self.t
        dt = b if b < a else a
        if self.hmin / smax < 1e-20:
            self.done = True
            return False
        self.local.advance_dt(dt)
        self.fresh = False
        self.t = self.t + dt
        self.steps += 1
        return True

    def advance(self, n: int) -> int:
        if self.on_device:
            before = self.steps
            self.enqueue_steps(n)
            return self.sync()[1] - before
        k = 0
        while k < n and self.step():
            k += 1
        return k

    def solve(self, check_every: int = 16) -> int:
        if self.on_device:
            before = self.steps
            while not self.done:
                self.enqueue_steps(check_every)
                self.sync()
            return self.steps - before
        k = 0
        while self.step():
            k += 1
        return k

    # ---- results -------------------------------------------------------------
    def owned_rows(self) -> np.ndarray:
        """This rank's rows [lo, hi) of the state, shape (hi-lo, nx, 4); the
        wrapped ghost rows of a periodic run are refreshed first.  Collective."""
        return np.ascontiguousarray(np.moveaxis(self.owned_planes(), 0, -1))

    def owned_planes(self, out: np.ndarray | None = None) -> np.ndarray:
        """As owned_rows, as planes (4, hi-lo, nx), into `out` if given (a
        pinned buffer makes the download fast).  Collective."""
        if not self.fresh:
            if self.on_device:
                import torch

                with torch.cuda.stream(self._stream):
                    self._exchange_on_stream()
                self.sync()
            else:
                self.exchange()
            self.fresh = True
        return self.local.get_rows(self.lo - self.l_lo, self.hi - self.lo, out=out)

    def conserved_totals(self) -> np.ndarray:
        """Mass, x momentum, y momentum and energy of the whole problem's
        interior, in FP64 (fvm2d_get_conserved_totals): each rank's solver
        sums its interior rows, which are exactly the rank's own rows inside
        the problem's ghost rows (its first and last two rows are halo or
        ghost rows), and the ranks' totals are added by an all-reduce.  The
        sum over ranks rounds differently from one device's.  Collective."""
        import torch

        v = torch.tensor(np.asarray(self.local.conserved_totals(), dtype=np.float64),
                         device="cuda" if self.device else "cpu")
        self.dist.all_reduce(v, op=self.dist.ReduceOp.SUM, group=self.group)
        return v.cpu().numpy()

    def gather(self) -> np.ndarray | None:
        """The whole state on rank 0 (None elsewhere).  Collective."""
        import torch

        mine = torch.from_numpy(self.owned_rows())
        if self.device:
            mine = mine.cuda()
        if self.rank != 0:
            self.dist.send(mine, self._global(0), group=self.group)
            return None
        out = np.empty((self.ny, self.nx, 4))
        out[self.lo:self.hi] = mine.cpu().numpy()
        for r, (lo, hi) in enumerate(plan_slabs(self.ny, self.world)):
            if r == 0:
                continue
            buf = torch.empty((hi - lo, self.nx, 4), dtype=torch.float64, device=mine.device)
            self.dist.recv(buf, self._global(r), group=self.group)
            out[lo:hi] = buf.cpu().numpy()
        return out

    def close(self) -> None:
        self.local.close()
