"""GPU error metrics (double-double, one warp per matrix) against exact rational
arithmetic on small matrices and against the reference's long-double metrics
(via the oracle) on large ones."""
import numpy as np
import pytest

from conftest import load_pkg
from oracle import exact_metrics as X

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

device = load_pkg("device")
M = load_pkg("matrices")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("n", [1, 2, 5, 9])
def test_metrics_match_exact_arithmetic(oracle, n):
    r = np.random.default_rng(n)
    A = M.general(r, 6, n, 1e3)
    S = M.spd(r, 6, n, 1e3)
    b = r.standard_normal((6, n))
    x = np.linalg.solve(A, b[..., None])[..., 0] * (1 + 1e-13 * r.standard_normal((6, n)))
    LU, piv, _ = oracle.lu(A, "scalar")
    L, _ = oracle.cholesky(S, "simd")
    got = device.solve_backward_error(dev(A), dev(x), dev(b)).cpu().numpy()
    np.testing.assert_allclose(got, X.solve_backward_error(A, x, b), rtol=1e-13, atol=0)
    got = device.lu_backward_error(dev(A), dev(LU), dev(piv.astype(np.int32))).cpu().numpy()
    np.testing.assert_allclose(got, X.lu_backward_error(A, LU, piv), rtol=1e-13, atol=0)
    got = device.chol_backward_error(dev(S), dev(L)).cpu().numpy()
    np.testing.assert_allclose(got, X.chol_backward_error(S, L), rtol=1e-13, atol=0)


def test_exact_cases():
    A = np.eye(4)[None].repeat(3, 0)
    b = np.arange(12.0).reshape(3, 4) + 1
    assert (device.solve_backward_error(dev(A), dev(b), dev(b)).cpu().numpy() == 0).all()
    piv = np.tile(np.arange(4, dtype=np.int32), (3, 1))
    assert (device.lu_backward_error(dev(A), dev(A), dev(piv)).cpu().numpy() == 0).all()
    assert (device.chol_backward_error(dev(A), dev(A)).cpu().numpy() == 0).all()


@pytest.mark.parametrize("n", [33, 64])
def test_metrics_agree_with_long_double(oracle, n):
    r = np.random.default_rng(100 + n)
    A = M.general(r, 40, n, M.log_uniform(r, 40, 1e1, 1e10))
    S = M.spd(r, 40, n, M.log_uniform(r, 40, 1e1, 1e10))
    b = r.standard_normal((40, n))
    LU, piv, _ = oracle.lu(A, "scalar")
    x = oracle.lu_solve(LU, piv, b[..., None])[..., 0]
    L, _ = oracle.cholesky(S, "simd")
    # the long double's 64-bit sums carry a few percent of error on residuals this
    # close to the unit roundoff; double-double does not
    g = device.solve_backward_error(dev(A), dev(x), dev(b)).cpu().numpy()
    np.testing.assert_allclose(g, oracle.solve_backward_error(A, x, b), rtol=0.05)
    g = device.lu_backward_error(dev(A), dev(LU), dev(piv.astype(np.int32))).cpu().numpy()
    np.testing.assert_allclose(g, oracle.lu_backward_error(A, LU, piv), rtol=0.05)
    g = device.chol_backward_error(dev(S), dev(L)).cpu().numpy()
    np.testing.assert_allclose(g, oracle.chol_backward_error(S, L), rtol=0.05)
    # and exactly where the exact checker is affordable
    np.testing.assert_allclose(device.lu_backward_error(dev(A[:2]), dev(LU[:2]), dev(piv[:2].astype(np.int32)))
                               .cpu().numpy(), X.lu_backward_error(A[:2], LU[:2], piv[:2]), rtol=1e-12)


def test_metric_errors():
    z = torch.zeros(2, 65, 65, dtype=torch.float64, device="cuda")
    v = torch.zeros(2, 65, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        device.solve_backward_error(z, v, v)
    with pytest.raises(TypeError):
        device.chol_backward_error(z[:, :4, :4].contiguous().float(), z[:, :4, :4].contiguous())
