"""The NumPy-facing drop-in API on its CPU backends, mirroring TinySolverDx's own
Python tests (tests/python/test_solvers.py), plus bit-for-bit agreement of every
CPU backend with the oracle (itself pinned to the compiled reference)."""
import numpy as np
import pytest
import scipy.linalg as sla

from conftest import load_pkg

tsdx = load_pkg()
matrices = load_pkg("matrices")

SIZES = [2, 3, 5, 8, 16, 17, 32, 64]
BACKENDS = ["naive", "scalar", "simd", "auto"]


def rng(seed=0):
    return np.random.default_rng(seed)


def bits_equal(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    iv = np.uint64 if a.dtype == np.float64 else np.uint32
    return np.array_equal(a.view(iv), b.view(iv))


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("backend", BACKENDS)
@pytest.mark.parametrize("dtype,tol", [(np.float64, 1e-12), (np.float32, 1e-4)])
def test_cholesky_matches_numpy(n, backend, dtype, tol):
    A = matrices.spd(rng(n), 21, n, 1e2).astype(dtype)
    L, info = tsdx.cholesky(A, backend=backend)
    assert L.dtype == dtype and (info == 0).all()
    np.testing.assert_allclose(L, np.linalg.cholesky(A.astype(np.float64)), atol=tol, rtol=tol)
    assert np.allclose(np.triu(L, 1), 0)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("backend", BACKENDS)
def test_lu_matches_scipy(n, backend):
    A = matrices.general(rng(n), 13, n, 1e3)
    LU, piv, info = tsdx.lu(A, backend=backend)
    assert (info == 0).all()
    for b in range(A.shape[0]):
        ref_lu, ref_piv = sla.lu_factor(A[b])
        np.testing.assert_array_equal(piv[b], ref_piv)
        np.testing.assert_allclose(LU[b], ref_lu, atol=1e-10, rtol=1e-10)


@pytest.mark.parametrize("n", [2, 7, 32, 64])
def test_solvers_match_numpy_solve(n):
    r = rng(1)
    A = matrices.general(r, 9, n, 1e3)
    S = matrices.spd(r, 9, n, 1e3)
    b = r.standard_normal((9, n))
    x, info = tsdx.gesv(A, b)
    np.testing.assert_allclose(x, np.linalg.solve(A, b[..., None])[..., 0], rtol=1e-8, atol=1e-8)
    x, info = tsdx.posv(S, b)
    assert (info == 0).all()
    np.testing.assert_allclose(x, np.linalg.solve(S, b[..., None])[..., 0], rtol=1e-8, atol=1e-8)
    B = r.standard_normal((9, n, 3))
    x, _ = tsdx.gesv(A, B)
    np.testing.assert_allclose(A @ x, B, atol=1e-9)


def test_single_matrix_and_vector_rhs():
    A = matrices.spd(rng(), 1, 6, 10.0)[0]
    b = np.arange(6.0)
    x, info = tsdx.posv(A, b)
    assert x.shape == (6,) and info == 0
    np.testing.assert_allclose(x, np.linalg.solve(A, b), atol=1e-12)
    x, info = tsdx.gesv(A, b)
    np.testing.assert_allclose(x, np.linalg.solve(A, b), atol=1e-12)


def test_input_not_modified_and_noncontiguous():
    A = matrices.spd(rng(), 4, 8, 10.0)
    keep = A.copy()
    tsdx.cholesky(A)
    np.testing.assert_array_equal(A, keep)
    big = np.zeros((4, 8, 16))
    big[:, :, ::2] = A
    L, _ = tsdx.cholesky(big[:, :, ::2])
    np.testing.assert_allclose(L, np.linalg.cholesky(A), atol=1e-12)


def test_not_positive_definite_reports_info():
    A = matrices.spd(rng(), 3, 5, 10.0)
    A[1] = -np.eye(5)
    _, info = tsdx.cholesky(A)
    assert list(info) == [0, 1, 0]


def test_singular_lu_reports_info():
    A = matrices.general(rng(), 2, 4, 10.0)
    _, _, info = tsdx.lu(A)
    assert list(info) == [0, 0]
    A[1] = 0
    _, _, info = tsdx.lu(A)
    assert info[1] == 1


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_emulated_precisions_have_expected_accuracy(prec):
    u = tsdx.unit_roundoff(prec)
    A = tsdx.round_to(matrices.spd(rng(3), 20, 16, 10.0), prec)
    L, info = tsdx.cholesky(A.astype(np.float32), precision=prec)
    assert (info == 0).all()
    assert (tsdx.round_to(L, prec) == L).all()
    err = tsdx.chol_backward_error(A, L.astype(np.float64))
    assert err.max() < 20 * u * 16 and err.max() > tsdx.unit_roundoff("fp32")


def test_float16_dtype_roundtrip():
    A = matrices.spd(rng(), 5, 8, 10.0).astype(np.float16)
    L, info = tsdx.cholesky(A)
    assert L.dtype == np.float16 and (info == 0).all()


def test_errors():
    with pytest.raises(ValueError):
        tsdx.cholesky(np.zeros((1, 65, 65), np.float64))
    with pytest.raises(ValueError):
        tsdx.cholesky(np.zeros((1, 3, 4), np.float64))
    with pytest.raises(ValueError):
        tsdx.cholesky(np.eye(3)[None], precision="fp8")
    with pytest.raises(TypeError):
        tsdx.cholesky(np.eye(3, dtype=np.int32))
    with pytest.raises(ValueError):
        tsdx.cholesky(np.eye(3)[None], backend="tpu")
    if not tsdx.has_cuda():
        with pytest.raises(RuntimeError):
            tsdx.cholesky(np.eye(3)[None], backend="cuda")
        with pytest.raises(RuntimeError):
            tsdx.gesv(np.eye(3)[None], np.ones((1, 3)), backend="cuda")
    # emulated formats on backend="cuda" need a device (the GPU emulation is checked
    # bit for bit against the CPU path in test_gpu_emu.py)
    if not tsdx.has_cuda():
        with pytest.raises(RuntimeError):
            tsdx.cholesky(np.eye(3, dtype=np.float32)[None], precision="bf16", backend="cuda")


def test_error_metrics_against_numpy():
    r = rng(5)
    A = matrices.general(r, 6, 10, 1e4)
    b = r.standard_normal((6, 10))
    LU, piv, _ = tsdx.lu(A)
    assert tsdx.lu_backward_error(A, LU, piv).max() < 1e-14
    x = np.linalg.solve(A, b[..., None])[..., 0]
    assert tsdx.solve_backward_error(A, x, b).max() < 1e-14
    assert tsdx.solve_forward_error(A, x, b).max() < 1e-10
    np.testing.assert_allclose(tsdx.reference_solve(A, b), x, rtol=1e-9)
    assert tsdx.solve_forward_error(A, x * 1.01, b).min() > 5e-3


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 9, 16, 17, 24, 25, 33, 64])
def test_cpu_backends_bit_exact_with_oracle(oracle, n, dtype):
    r = rng(70 + n)
    G = r.standard_normal((11, n, n)).astype(dtype)
    if n > 2:
        G[2, :, 1] = 0
        G[4] = r.integers(-2, 3, (n, n))
    S = (G @ G.transpose(0, 2, 1) + n * np.eye(n)).astype(dtype)
    if n > 3:
        S[5, 2, 2] = -1
    B = r.standard_normal((11, n, 3)).astype(dtype)
    for be in BACKENDS:
        LU, piv, info = tsdx.lu(G, backend=be)
        LUo, pivo, infoo = oracle.lu(G, be)
        assert bits_equal(LU, LUo) and np.array_equal(piv, pivo) and np.array_equal(info, infoo), be
        L, cinfo = tsdx.cholesky(S, backend=be)
        Lo, cinfoo = oracle.cholesky(S, be)
        ok = cinfoo == 0
        assert np.array_equal(cinfo, cinfoo) and bits_equal(L[ok], Lo[ok]), be
    Lo, _ = oracle.cholesky((G @ G.transpose(0, 2, 1) + n * np.eye(n)).astype(dtype), "simd")
    assert bits_equal(tsdx.cholesky_solve(Lo, B), oracle.cholesky_solve(Lo, B))
    LUo, pivo, _ = oracle.lu(G, "scalar")
    assert bits_equal(tsdx.lu_solve(LUo, pivo, B), oracle.lu_solve(LUo, pivo, B))


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
def test_emulated_bit_exact_with_oracle(oracle, prec):
    r = rng(8)
    for n in (2, 5, 16, 33):
        S = matrices.spd(r, 5, n, 10.0)
        L, info = tsdx.cholesky(S, precision=prec)
        Lo, infoo = oracle.emu_cholesky(prec, S)
        assert bits_equal(L, Lo) and np.array_equal(info, infoo)
        G = r.standard_normal((5, n, n))
        LU, piv, info = tsdx.lu(G, precision=prec)
        LUo, pivo, infoo = oracle.emu_lu(prec, G)
        assert bits_equal(LU, LUo) and np.array_equal(piv, pivo)
        x = r.standard_normal((5, n, 2))
        assert bits_equal(tsdx.lu_solve(LUo, pivo, x, precision=prec), oracle.emu_lu_solve(prec, LUo, pivo, x))


def test_metrics_bit_exact_with_oracle(oracle, golden):
    A, b, x = golden["metric_A"], golden["metric_b"], golden["metric_x"]
    LU, piv, _ = oracle.lu(A, "auto")
    assert bits_equal(tsdx.lu_backward_error(A, LU, piv), golden["metric_lu_bwd"])
    assert bits_equal(tsdx.solve_backward_error(A, x, b), golden["metric_solve_bwd"])
    assert bits_equal(tsdx.solve_forward_error(A, x, b), golden["metric_solve_fwd"])
    assert bits_equal(tsdx.reference_solve(A, b), golden["metric_xref"])
    S = golden["metric_S"]
    L, _ = oracle.cholesky(S, "auto")
    assert bits_equal(tsdx.chol_backward_error(S, L), golden["metric_chol_bwd"])
