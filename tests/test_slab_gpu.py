"""Row slabs on the GPU: two or three processes share the one GPU, each with
its own libfvm2d solver holding a slab plus halo rows, exchanging rows
through host memory between steps (gloo).  The gathered result must equal a
single solver's run of the whole array bit for bit, including the presets
whose ghost rules use global row numbers (jet rows, the double-Mach shock
position), in the FP64, FP32 and residual builds (the rows carry hi + lo).  The NCCL path, whose steps are enqueued on the device with no
host round trip (asynchronous row transfers, device-side max reduction and
step plan), runs as one rank on the one GPU and must equal the single
solver bit for bit too."""
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import slab_ranks

pytestmark = pytest.mark.gpu


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def single(pkg, case):
    U = pkg.scenarios.seeded_four_quadrant(case["nx"], case["ny"], case["seed"])
    h = pkg.Handle(case["nx"], case["ny"])
    h.configure(case["width"], case["height"], case["t_end"], 0.45, 1.9, 1.4, case["strategy"], case["precision"])
    h.set_state(U)
    h.solve()
    t, steps, _ = h.time()
    V = h.get_state(4)
    h.close()
    return V, t, steps


CASES = [dict(world=w, nx=48, ny=53, seed=10 + s, strategy=s, width=1.0, height=1.1, t_end=0.03, precision=p)
         for w, s, p in [(2, 0, 1), (3, 2, 1), (2, 3, 1), (3, 4, 1), (3, 5, 1), (2, 6, 0), (2, 1, 4)]]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"world{c['world']}-strategy{c['strategy']}-prec{c['precision']}")
def test_gpu_slabs_equal_single_solver(pkg, case, tmp_path):
    out = str(tmp_path / "gathered.npz")
    mp.spawn(slab_ranks.gpu_worker, args=(case["world"], free_port(), case, out), nprocs=case["world"], join=True)
    z = np.load(out)
    G, t, steps = z["G"], float(z["t"]), int(z["steps"])
    V, vt, vsteps = single(pkg, case)
    assert (steps, t) == (vsteps, vt)
    assert np.array_equal(G, V, equal_nan=True)


@pytest.mark.parametrize("precision", [0, 3, 4])
def test_rows_round_trip_through_host_and_device_memory(pkg, precision):
    import torch

    nx, ny = 37, 29
    U = pkg.scenarios.seeded_four_quadrant(nx, ny, 7)
    h = pkg.Handle(nx, ny)
    h.configure(1.0, 1.0, 0.1, 0.45, 1.9, 1.4, 0, precision)
    h.set_state(U)
    S = h.get_state(4)
    R = h.get_rows(5, 3)
    assert np.array_equal(R, np.moveaxis(S[5:8], -1, 0))
    D = torch.empty((4, 2, nx), dtype=torch.float64, device="cuda")
    h.get_rows_ptr(20, 2, D.data_ptr())
    assert np.array_equal(D.cpu().numpy(), np.moveaxis(S[20:22], -1, 0))
    h.set_rows_ptr(0, 2, D.data_ptr())  # rows 20, 21 copied onto rows 0, 1 through device memory
    h.set_rows(10, R)                   # rows 5..7 onto rows 10..12 through host memory
    T = h.get_state(4)
    assert np.array_equal(T[0:2], S[20:22]) and np.array_equal(T[10:13], S[5:8])
    assert np.array_equal(T[2:10], S[2:10]) and np.array_equal(T[13:], S[13:])
    h.close()


NCCL_CASES = [dict(world=1, nx=96, ny=80, seed=3, strategy=s, width=1.0, height=0.9, t_end=0.05, precision=p, first=7)
              for s, p in [(0, 0), (5, 0), (4, 3), (2, 1), (6, 4)]]


@pytest.mark.parametrize("case", NCCL_CASES, ids=lambda c: f"strategy{c['strategy']}-prec{c['precision']}")
def test_device_enqueued_slab_steps_over_nccl_equal_single_solver(pkg, case, tmp_path):
    out = str(tmp_path / "gathered.npz")
    mp.spawn(slab_ranks.nccl_worker, args=(case["world"], free_port(), case, out), nprocs=case["world"], join=True)
    z = np.load(out)
    G, t, steps = z["G"], float(z["t"]), int(z["steps"])
    assert int(z["first"]) == case["first"]
    V, vt, vsteps = single(pkg, case)
    assert (steps, t) == (vsteps, vt)
    assert np.array_equal(G, V, equal_nan=True)


def test_async_row_transfers_refuse_host_memory(pkg):
    nx, ny = 40, 30
    h = pkg.Handle(nx, ny)
    h.configure(1.0, 1.0, 0.1, 0.45, 1.9, 1.4, 0, 0)
    h.set_state(pkg.scenarios.seeded_four_quadrant(nx, ny, 1))
    host = np.zeros((4, 2, nx))
    with pytest.raises(pkg.FVM2DError):
        h.get_rows_async(0, 2, host.ctypes.data)
    h.close()
