"""The FP64 product build divides and takes square roots through its own
refined reciprocals (fvm2d_math.cuh: the hardware's approximate seeds plus
one third-order step) instead of IEEE division.  Their error bound, checked
on the GPU against correctly rounded values computed on the host in extended
precision: at most 2 ulp over arguments spanning the exponent range the
solver meets, and exact powers of two.  fvm2d_eval_reciprocals runs the same
inline functions the sweep kernels run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ulp_error(got, exact_ld):
    exact = exact_ld.astype(np.float64)
    return np.abs(got.astype(np.longdouble) - exact_ld) / np.spacing(np.abs(exact)).astype(np.longdouble)


def test_refined_reciprocals_within_two_ulp(pkg):
    torch = pytest.importorskip("torch")
    lib = pkg.load()
    rng = np.random.default_rng(11)
    x = np.concatenate([
        np.exp(rng.uniform(np.log(1e-12), np.log(1e12), 400_000)),  # densities, pressures, c, products
        rng.uniform(0.5, 2.0, 200_000),                             # near one, all mantissas
        2.0 ** np.arange(-60, 61),                                   # exact powers of two
    ])
    xd = torch.from_numpy(x).cuda()
    r = torch.empty_like(xd)
    q = torch.empty_like(xd)
    assert lib.fvm2d_eval_reciprocals(xd.data_ptr(), x.size, r.data_ptr(), q.data_ptr()) == 0
    r, q = r.cpu().numpy(), q.cpu().numpy()
    xl = x.astype(np.longdouble)
    e_rcp = ulp_error(r, 1 / xl)
    e_rsq = ulp_error(q, 1 / np.sqrt(xl))
    print(f"max ulp: rcp {float(e_rcp.max()):.3f}, rsqrt {float(e_rsq.max()):.3f}; "
          f"mean: {float(e_rcp.mean()):.3f}, {float(e_rsq.mean()):.3f}")
    assert float(e_rcp.max()) <= 2.0
    assert float(e_rsq.max()) <= 2.0
    p2 = slice(600_000, None)
    assert np.array_equal(r[p2], 1.0 / x[p2])  # powers of two: exact

