"""The C oracle against the golden fixtures made by the reference's own kernels
(tests/golden/make_golden.py): bit-exact, NaN positions included."""
import numpy as np
import pytest

from oracle import OUTFLOW

SMALL = ["quad_outflow_48x32", "quad_reflective_32x48", "quad_outflow_alpha1_64x64", "double_mach_16",
         "jet_32", "jet800_16", "four_shocks_64", "four_contacts_48", "sedov_32", "quad_gamma5_3_32x32"]
RUN_KEYS = ("width", "height", "cfl", "alpha", "gamma", "t_end", "strategy")


@pytest.mark.parametrize("name", SMALL)
def test_oracle_matches_reference_fixture(oracle, golden, name):
    z, manifest = golden
    m = manifest[name]
    U1, steps, t = oracle.solve(z[f"{name}/U0"], max_steps=m["max_steps"], **{k: m[k] for k in RUN_KEYS})
    assert steps == m["steps"]
    assert t == m["t"]
    assert np.array_equal(U1, z[f"{name}/U1"], equal_nan=True)


def test_oracle_full_size_quadrant_checksums(oracle, golden, pkg):
    """400x400 seeded four-quadrant problem to t = 0.2 (620 steps): every step's
    time and per-field sums equal the reference's."""
    z, manifest = golden
    name = "quad_outflow_400x400_seed0"
    m = manifest[name]
    assert m["strategy"] == OUTFLOW
    U = pkg.scenarios.seeded_four_quadrant(m["nx"], m["ny"], m["seed"])
    times, sums = z[f"{name}/t"], z[f"{name}/field_sums"]
    t = 0.0
    for k in range(m["steps"]):
        r = oracle.step(U, t=t, **{key: m[key] for key in RUN_KEYS})
        assert r is not None, f"loop ended early at step {k}"
        U, t, _ = r
        assert t == times[k]
        assert np.array_equal(U.sum(axis=(0, 1)), sums[k])
    assert oracle.step(U, t=t, **{key: m[key] for key in RUN_KEYS}) is None
    assert np.array_equal(U[200], z[f"{name}/U1_row_200"])
    assert np.array_equal(U[:, 137], z[f"{name}/U1_col_137"])
