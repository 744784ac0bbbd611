"""The drop-in API with backend="cuda": same answers as the reference's CPU
backends (factors, pivots and info bit-for-bit; solutions to c*n*u), and the
torch-tensor device API."""
import numpy as np
import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

tsdx = load_pkg()
matrices = load_pkg("matrices")
device = load_pkg("device")


def bits_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    iv = np.uint64 if a.dtype == np.float64 else np.uint32
    return np.array_equal(a.view(iv), b.view(iv))


def test_has_cuda():
    assert tsdx.has_cuda()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [2, 5, 16, 17, 32, 64])
def test_cuda_factors_equal_cpu_backends(n, dtype):
    r = np.random.default_rng(n)
    A = matrices.general(r, 33, n, 1e4).astype(dtype)
    S = matrices.spd(r, 33, n, 1e3).astype(dtype)
    LU, piv, info = tsdx.lu(A, backend="cuda")
    LUc, pivc, infoc = tsdx.lu(A, backend="scalar")
    assert bits_equal(LU, LUc) and np.array_equal(piv, pivc) and np.array_equal(info, infoc)
    L, cinfo = tsdx.cholesky(S, backend="cuda")
    Lc, cinfoc = tsdx.cholesky(S, backend="simd")
    assert bits_equal(L, Lc) and np.array_equal(cinfo, cinfoc)


@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 2e-4)])
@pytest.mark.parametrize("n", [3, 16, 33, 64])
def test_cuda_solves(n, dtype, tol):
    r = np.random.default_rng(100 + n)
    A = matrices.general(r, 21, n, 1e2).astype(dtype)
    S = matrices.spd(r, 21, n, 1e2).astype(dtype)
    b = r.standard_normal((21, n)).astype(dtype)
    B = r.standard_normal((21, n, 10)).astype(dtype)
    ref = np.linalg.solve(A.astype(np.float64), b[..., None].astype(np.float64))[..., 0]
    x, info = tsdx.gesv(A, b, backend="cuda")
    assert (info == 0).all() and x.shape == b.shape
    np.testing.assert_allclose(x, ref, rtol=tol * 100, atol=tol * 100)
    x, info = tsdx.posv(S, B, backend="cuda")
    np.testing.assert_allclose(S.astype(np.float64) @ x, B, atol=tol * 100)
    L, _ = tsdx.cholesky(S, backend="cuda")
    np.testing.assert_allclose(tsdx.cholesky_solve(L, B, backend="cuda"), tsdx.cholesky_solve(L, B), rtol=tol * 100,
                               atol=tol * 100)
    LU, piv, _ = tsdx.lu(A, backend="cuda")
    np.testing.assert_allclose(tsdx.lu_solve(LU, piv, B, backend="cuda"), tsdx.lu_solve(LU, piv, B), rtol=tol * 100,
                               atol=tol * 100)


def test_single_matrix_and_inputs_untouched():
    A = matrices.spd(np.random.default_rng(), 1, 6, 10.0)[0]
    keep = A.copy()
    b = np.arange(6.0)
    x, info = tsdx.posv(A, b, backend="cuda")
    assert x.shape == (6,) and info == 0
    np.testing.assert_allclose(x, np.linalg.solve(A, b), atol=1e-12)
    x, info = tsdx.gesv(A, b, backend="cuda")
    np.testing.assert_allclose(x, np.linalg.solve(A, b), atol=1e-12)
    np.testing.assert_array_equal(A, keep)


def test_ir_python_api(oracle):
    r = np.random.default_rng(9)
    A = matrices.general(r, 64, 64, matrices.log_uniform(r, 64, 1e1, 1e12))
    b = r.standard_normal((64, 64))
    x, info, status, bwd = tsdx.gesv_ir(A, b, tier="fp32")
    xp, _ = tsdx.gesv(A, b, backend="cuda")
    assert oracle.solve_backward_error(A, x, b).max() <= 2 * oracle.solve_backward_error(A, xp, b).max() + 2.0 ** -53
    assert ((status >= 0) | (status == -1)).all()
    S = matrices.spd(r, 16, 32, 1e3)
    x, info, status, bwd = tsdx.posv_ir(S, b[:16, :32], tier=np.full(16, 2, np.int8))
    assert (status >= 0).all()


def test_device_tensor_api():
    r = np.random.default_rng(5)
    A = torch.from_numpy(matrices.general(r, 50, 40, 1e3)).cuda()
    B = torch.randn(50, 40, 3, dtype=torch.float64, device="cuda")
    A0, B0 = A.clone(), B.clone()
    piv, info = device.gesv(A, B)
    assert (info == 0).all()
    torch.testing.assert_close(A0 @ B, B0, atol=1e-9, rtol=0)
    S = A0 @ A0.transpose(1, 2) + 40 * torch.eye(40, dtype=torch.float64, device="cuda")
    X = B0.clone()
    info = device.posv(S.clone(), X)
    torch.testing.assert_close(S @ X, B0, atol=1e-9, rtol=0)
