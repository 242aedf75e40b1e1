"""The C oracle against the reference's own kernels compiled for the host
(oracle/_ref/libref_host.so) on fresh seeded cases: bit-exact.  Skipped where
the reference was not available at build time."""
import numpy as np
import pytest

from oracle import RefHost

pytestmark = pytest.mark.skipif(not RefHost.available(), reason="oracle/_ref not built (reference sources absent)")


@pytest.mark.parametrize("strategy", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("seed", [11, 12])
def test_oracle_equals_reference_host_build(oracle, pkg, strategy, seed):
    nx, ny = (64, 32) if seed % 2 else (32, 48)
    U0 = pkg.scenarios.seeded_four_quadrant(nx, ny, seed * 10 + strategy)
    kw = dict(width=1.0 + 0.25 * strategy, height=0.75, cfl=0.45, alpha=1.2 + 0.2 * strategy, gamma=1.4,
              t_end=0.03, strategy=strategy)
    A, sa, ta = oracle.solve(U0, max_steps=12, **kw)
    B, sb, tb = RefHost().run(U0, max_steps=12, **kw)
    assert (sa, ta) == (sb, tb)
    assert np.array_equal(A, B, equal_nan=True)


def test_y_sweep_of_x_only_state_is_a_round_trip(oracle):
    """A state varying only along x has zero y-slopes and zero y-flux
    differences, so a y-sweep only round-trips primitive -> conserved ->
    primitive (ulp-level changes, src/basicFuns.cuh:240-244)."""
    U = np.zeros((16, 32, 4))
    x = np.linspace(0, 1, 32)
    U[:, :, 0] = 1 + 0.2 * np.sin(2 * np.pi * x)
    U[:, :, 1] = 1.0
    U[:, :, 2] = 0.3
    V = oracle.sweep_y(U, height=1.0, dt=1e-3)
    assert np.abs(V - U).max() < 1e-14
    assert np.array_equal(U[..., 0], V[..., 0])
