"""Generates tests/golden/reference_cases.npz from the reference's own kernels.

Run in a checkout where the reference sources were available at build time:
    make -C oracle ref && python tests/golden/make_golden.py

Every case is executed by oracle/_ref/libref_host.so: the reference's
src/basicFuns.cuh and src/ghostCellPresets.cuh compiled unchanged for the
host and driven in the launch order of src/wrappers.cuh:154-306, with
contraction off.  The fixture stores, per case, the parameters, the initial
state, the state after the run, the step count and the final time; the
full-size four-quadrant case (400x400, the reference-parity workload) stores
per-step times and field sums instead of states to stay small.
"""
from __future__ import annotations

import importlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
from oracle import RefHost, OUTFLOW, REFLECTIVE, JET, JET800, DOUBLE_MACH  # noqa: E402

sc = importlib.import_module("2d_fvm_cuda_b200.scenarios")

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_cases.npz")

# name -> (initial state, run parameters)
CASES = {
    "quad_outflow_48x32": (sc.seeded_four_quadrant(48, 32, 101),
                           dict(width=1.0, height=1.0, cfl=0.45, alpha=1.9, gamma=1.4, t_end=0.05, strategy=OUTFLOW)),
    "quad_reflective_32x48": (sc.seeded_four_quadrant(32, 48, 102),
                              dict(width=1.0, height=1.5, cfl=0.45, alpha=1.9, gamma=1.4, t_end=0.03, strategy=REFLECTIVE)),
    "quad_outflow_alpha1_64x64": (sc.seeded_four_quadrant(64, 64, 103),
                                  dict(width=1.0, height=1.0, cfl=0.5, alpha=1.0, gamma=1.4, t_end=0.04, strategy=OUTFLOW)),
    "double_mach_16": (sc.double_mach(16),
                       dict(width=4.0, height=1.0, cfl=0.45, alpha=1.9, gamma=1.4, t_end=0.02, strategy=DOUBLE_MACH)),
    "jet_32": (sc.jet(32),
               dict(width=2.0, height=1.0, cfl=0.45, alpha=1.9, gamma=1.4, t_end=1.0, strategy=JET, max_steps=25)),
    "jet800_16": (sc.jet800(16),
                  dict(width=3.0, height=1.0, cfl=0.45, alpha=1.9, gamma=1.4, t_end=1.0, strategy=JET800, max_steps=25)),
    "four_shocks_64": (sc.four_shocks(64),
                       dict(width=1.0, height=1.0, cfl=0.5, alpha=2.0, gamma=1.4, t_end=0.1, strategy=OUTFLOW)),
    "four_contacts_48": (sc.four_contacts(48),
                         dict(width=1.0, height=1.0, cfl=0.5, alpha=1.7, gamma=1.4, t_end=0.1, strategy=OUTFLOW)),
    "sedov_32": (sc.sedov_1d(32),
                 dict(width=8.0, height=8.0, cfl=0.45, alpha=1.9, gamma=1.4, t_end=1.0, strategy=OUTFLOW, max_steps=30)),
    "quad_gamma5_3_32x32": (sc.seeded_four_quadrant(32, 32, 104),
                            dict(width=1.0, height=1.0, cfl=0.4, alpha=1.5, gamma=5.0 / 3.0, t_end=0.05, strategy=OUTFLOW)),
}

# The reference-parity workload: 400x400 incl. ghosts on [0,1]^2, gamma 1.4,
# transmissive, CFL 0.45, t_end 0.2, seeded four-quadrant data, alpha 1.9.
FULL = ("quad_outflow_400x400_seed0", 400, 400, 0,
        dict(width=1.0, height=1.0, cfl=0.45, alpha=1.9, gamma=1.4, t_end=0.2, strategy=OUTFLOW))


def main() -> None:
    ref = RefHost()
    arrays = {}
    manifest = {}
    for name, (U0, kw) in CASES.items():
        kw = dict(kw)
        max_steps = kw.pop("max_steps", -1)
        U1, steps, t = ref.run(U0, max_steps=max_steps, **kw)
        arrays[f"{name}/U0"] = U0
        arrays[f"{name}/U1"] = U1
        manifest[name] = dict(kw, max_steps=max_steps, steps=steps, t=t)
        print(f"{name}: {steps} steps to t={t!r}")

    name, nx, ny, seed, kw = FULL
    U = sc.seeded_four_quadrant(nx, ny, seed)
    times, sums = [], []
    t = 0.0
    while True:
        U, k, t_new = ref.run(U, t0=t, max_steps=1, **kw)
        if k == 0:
            break
        t = t_new
        times.append(t)
        sums.append(U.sum(axis=(0, 1)))
    arrays[f"{name}/t"] = np.array(times)
    arrays[f"{name}/field_sums"] = np.array(sums)
    arrays[f"{name}/U1_row_200"] = U[200].copy()
    arrays[f"{name}/U1_col_137"] = U[:, 137].copy()
    manifest[name] = dict(kw, nx=nx, ny=ny, seed=seed, steps=len(times), t=t)
    print(f"{name}: {len(times)} steps to t={t!r}")

    arrays["manifest"] = np.frombuffer(json.dumps(manifest, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
