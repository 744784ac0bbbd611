"""GPU parity of the sm_100a kernels against the CPU oracle, through the C-ABI.

Factors, pivots and info must be bit-identical to the oracle (which is pinned
bit-for-bit to the compiled reference): LU to kernels.hpp:91-119 (scalar/simd
backends, identical), Cholesky to kernels.hpp:57-87 as the reference's default
simd backend compiles it. Solutions must meet a normwise backward error of
c*n*u (c = 8), the tolerance the reference's own tests use for its factors
(tests/cpp/test_solvers.cpp:58, :123), evaluated in float64.
"""
import numpy as np
import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

capi = load_pkg("capi")
M = load_pkg("matrices")

SIZES = [1, 2, 3, 4, 5, 7, 8, 9, 12, 15, 16, 17, 20, 23, 24, 25, 31, 32, 33, 39, 40, 41, 47, 48, 49,
         55, 56, 57, 63, 64]
U = {np.float32: 2.0 ** -24, np.float64: 2.0 ** -53}
C_BWD = 8.0


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    iv = np.uint64 if a.dtype == np.float64 else np.uint32
    return np.array_equal(a.view(iv), b.view(iv))


def lu_inputs(n, batch, dtype, seed):
    rng = np.random.default_rng(seed)
    A = M.general(rng, batch, n, M.log_uniform(rng, batch, 1e1, 1e4)).astype(dtype)
    if batch >= 8 and n >= 2:
        A[1, :, n // 2] = 0.0                                   # zeroed column -> info > 0
        A[2] = 0.0                                              # zero matrix -> info 1
        A[3] = rng.integers(-2, 3, (n, n)).astype(dtype)        # many exact ties in the argmax
        A[4, n - 1] = A[4, 0]                                   # duplicate rows
        A[5] = np.abs(rng.integers(0, 2, (n, n))).astype(dtype) # ties and zeros
    return A


def chol_inputs(n, batch, dtype, seed):
    rng = np.random.default_rng(seed)
    A = M.spd(rng, batch, n, M.log_uniform(rng, batch, 1e1, 1e3)).astype(dtype)
    if batch >= 8:
        A[1, n // 2, n // 2] = -1.0                             # not positive definite
        A[2] = 0.0                                              # info 1
        if n >= 2:
            A[3, n - 1, n - 1] = 0.0                            # breaks at the last pivot (usually)
    return A


def gpu_getrf(A):
    a = dev(A)
    piv = torch.zeros(A.shape[:2], dtype=torch.int32, device="cuda")
    info = torch.full((A.shape[0],), -7, dtype=torch.int32, device="cuda")
    capi.getrf(a, piv, info)
    return host(a), host(piv), host(info)


def gpu_potrf(A):
    a = dev(A)
    info = torch.full((A.shape[0],), -7, dtype=torch.int32, device="cuda")
    capi.potrf(a, info)
    return host(a), host(info)


def solve_bwd(A, X, B):
    """max over matrices and columns of ||b - A x|| / (||A||_F ||x|| + ||b||) in float64."""
    A = A.astype(np.float64)
    X = X.astype(np.float64)
    B = B.astype(np.float64)
    R = B - A @ X
    num = np.linalg.norm(R, axis=1)
    den = np.linalg.norm(A, axis=(1, 2))[:, None] * np.linalg.norm(X, axis=1) + np.linalg.norm(B, axis=1)
    return num / den


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", SIZES)
def test_getrf_bit_exact(oracle, n, dtype):
    A = lu_inputs(n, 37, dtype, 100 + n)
    LU, piv, info = gpu_getrf(A)
    LUo, pivo, infoo = oracle.lu(A, "scalar")
    np.testing.assert_array_equal(info, infoo)
    np.testing.assert_array_equal(piv, pivo)
    assert bits_equal(LU, LUo), np.abs(LU - LUo).max()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", SIZES)
def test_potrf_bit_exact(oracle, n, dtype):
    A = chol_inputs(n, 37, dtype, 200 + n)
    L, info = gpu_potrf(A)
    Lo, infoo = oracle.cholesky(A, "simd")
    np.testing.assert_array_equal(info, infoo)
    assert bits_equal(L, Lo), np.abs(L - Lo).max()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 5, 8, 16, 17, 32, 33, 48, 64])
@pytest.mark.parametrize("nrhs", [1, 3, 4, 8, 11])
def test_gesv(oracle, n, nrhs, dtype):
    A = lu_inputs(n, 37, dtype, 300 + n)
    rng = np.random.default_rng(n * 7 + nrhs)
    B = rng.standard_normal((37, n, nrhs)).astype(dtype)
    a, b = dev(A), dev(B)
    piv = torch.zeros((37, n), dtype=torch.int32, device="cuda")
    info = torch.zeros(37, dtype=torch.int32, device="cuda")
    capi.gesv(a, b, piv, info)
    LU, X, P, I = host(a), host(b), host(piv), host(info)
    LUo, Po, Xo, Io = oracle.gesv(A, B, "scalar")
    np.testing.assert_array_equal(I, Io)
    np.testing.assert_array_equal(P, Po)
    assert bits_equal(LU, LUo)
    ok = I == 0
    bwd = solve_bwd(A[ok], X[ok], B[ok])
    assert bwd.max() <= C_BWD * n * U[dtype], bwd.max()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 2, 5, 8, 16, 17, 32, 33, 48, 64])
@pytest.mark.parametrize("nrhs", [1, 3, 4, 8, 11])
def test_posv(oracle, n, nrhs, dtype):
    A = chol_inputs(n, 37, dtype, 400 + n)
    rng = np.random.default_rng(n * 11 + nrhs)
    B = rng.standard_normal((37, n, nrhs)).astype(dtype)
    a, b = dev(A), dev(B)
    info = torch.zeros(37, dtype=torch.int32, device="cuda")
    capi.posv(a, b, info)
    L, X, I = host(a), host(b), host(info)
    Lo, Xo, Io = oracle.posv(A, B, "simd")
    np.testing.assert_array_equal(I, Io)
    assert bits_equal(L, Lo)
    ok = I == 0
    bwd = solve_bwd(A[ok], X[ok], B[ok])
    assert bwd.max() <= C_BWD * n * U[dtype], bwd.max()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("n", [1, 3, 16, 31, 32, 33, 64])
@pytest.mark.parametrize("nrhs", [1, 2, 9])
def test_getrs_potrs(oracle, n, nrhs, dtype):
    rng = np.random.default_rng(n + 50 * nrhs)
    A = M.general(rng, 19, n, 1e3).astype(dtype)
    S = M.spd(rng, 19, n, 1e3).astype(dtype)
    B = rng.standard_normal((19, n, nrhs)).astype(dtype)
    LU, piv, _ = oracle.lu(A, "scalar")
    b = dev(B)
    capi.getrs(dev(LU), dev(piv), b)
    X = host(b)
    assert solve_bwd(A, X, B).max() <= C_BWD * n * U[dtype]
    np.testing.assert_allclose(X, oracle.lu_solve(LU, piv, B), rtol=1e-3 if dtype == np.float32 else 1e-9,
                               atol=1e-3 if dtype == np.float32 else 1e-9)
    L, _ = oracle.cholesky(S, "simd")
    b = dev(B)
    capi.potrs(dev(L), b)
    X = host(b)
    assert solve_bwd(S, X, B).max() <= C_BWD * n * U[dtype]


def test_golden_vectors(golden):
    """The committed fixtures (made by the reference itself) through the GPU path."""
    for key in golden.files:
        if not key.endswith("_gen"):
            continue
        k = key[:-4]
        A = golden[key]
        LU, piv, info = gpu_getrf(A)
        assert bits_equal(LU, golden[k + "_LU"]), k
        np.testing.assert_array_equal(piv, golden[k + "_piv"])
        np.testing.assert_array_equal(info, golden[k + "_luinfo"])
        L, cinfo = gpu_potrf(golden[k + "_spd"])
        assert bits_equal(L, golden[k + "_L"]), k
        np.testing.assert_array_equal(cinfo, golden[k + "_info"])
    LU, piv, info = gpu_getrf(golden["kat_pivot2"])
    assert list(piv[0]) == [1, 1] and info[0] == 0 and LU[0, 0, 0] == 1 and LU[0, 1, 1] == 1
    _, info = gpu_potrf(golden["kat_nonspd"])
    np.testing.assert_array_equal(info, golden["kat_nonspd_info"])
    _, piv, info = gpu_getrf(golden["kat_singular"])
    np.testing.assert_array_equal(info, golden["kat_singular_info"])
    np.testing.assert_array_equal(piv, golden["kat_singular_piv"])


@pytest.mark.parametrize("n,batch", [(4, 200_003), (16, 70_001), (64, 5_001)])
def test_large_batch_loops(oracle, n, batch):
    """Batches larger than one wave of resident warps exercise the persistent loop."""
    rng = np.random.default_rng(n)
    A = rng.standard_normal((batch, n, n))
    LU, piv, info = gpu_getrf(A)
    idx = rng.choice(batch, 512, replace=False)
    LUo, pivo, infoo = oracle.lu(A[idx], "scalar")
    assert bits_equal(LU[idx], LUo)
    np.testing.assert_array_equal(piv[idx], pivo)
    S = A @ A.transpose(0, 2, 1) + n * np.eye(n)
    L, info = gpu_potrf(S)
    Lo, _ = oracle.cholesky(S[idx], "simd")
    assert bits_equal(L[idx], Lo)
    assert (info == 0).all()


def test_nonfinite_inputs(oracle):
    """NaN/Inf propagate like the reference: NaN never wins a pivot search unless on the diagonal."""
    rng = np.random.default_rng(9)
    for n in (5, 17, 40):
        A = rng.standard_normal((12, n, n))
        A[0, 0, 0] = np.nan
        A[1, 3 % n, 0] = np.nan
        A[2, 1, 1] = np.inf
        A[3, :, 2] = np.nan
        LU, piv, info = gpu_getrf(A)
        LUo, pivo, infoo = oracle.lu(A, "scalar")
        np.testing.assert_array_equal(piv, pivo)
        np.testing.assert_array_equal(info, infoo)
        np.testing.assert_array_equal(np.isnan(LU), np.isnan(LUo))
        fin = np.isfinite(LUo)
        np.testing.assert_array_equal(LU[fin], LUo[fin])


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_host_pointer_api(oracle, dtype):
    """The synchronous host-pointer entry points (chunked, copies overlapped)."""
    lib = capi.lib()
    s = capi.sfx(np.dtype(dtype))
    for n, batch in ((16, 5000), (64, 7000), (33, 41)):
        A = lu_inputs(n, batch, dtype, n)
        B = np.random.default_rng(1).standard_normal((batch, n, 4)).astype(dtype)
        a, b = A.copy(), B.copy()
        piv = np.zeros((batch, n), np.int32)
        info = np.zeros(batch, np.int32)
        capi.check(getattr(lib, f"tsdx_cuda_gesv_batched_host_{s}")(capi.ptr(a), n, batch, capi.ptr(b), 4,
                                                                   capi.ptr(piv), capi.ptr(info)))
        LUo, pivo, infoo = oracle.lu(A, "scalar")
        assert bits_equal(a, LUo)
        np.testing.assert_array_equal(piv, pivo)
        np.testing.assert_array_equal(info, infoo)
        ok = info == 0
        assert solve_bwd(A[ok], b[ok], B[ok]).max() <= C_BWD * n * U[dtype]
        S = chol_inputs(n, batch, dtype, n + 1)
        l = S.copy()
        cinfo = np.zeros(batch, np.int32)
        capi.check(getattr(lib, f"tsdx_cuda_cholesky_batched_host_{s}")(capi.ptr(l), n, batch, capi.ptr(cinfo)))
        Lo, infoo = oracle.cholesky(S, "simd")
        assert bits_equal(l, Lo)
        np.testing.assert_array_equal(cinfo, infoo)


def test_argument_errors():
    a = torch.zeros((2, 3, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        capi.check(capi.call("tsdx_cuda_potrf_f64", capi.ptr(a), 65, 2, None, capi.stream_ptr()))
    with pytest.raises(ValueError):
        capi.check(capi.call("tsdx_cuda_potrf_f64", capi.ptr(a), 0, 2, None, capi.stream_ptr()))
    with pytest.raises(ValueError):
        capi.check(capi.call("tsdx_cuda_potrf_f64", capi.ptr(a), 3, -1, None, capi.stream_ptr()))
    with pytest.raises(ValueError):
        capi.check(capi.call("tsdx_cuda_getrf_f64", capi.ptr(a), 3, 2, None, None, capi.stream_ptr()))
    assert capi.call("tsdx_cuda_potrf_f64", capi.ptr(a), 3, 0, None, capi.stream_ptr()) == 0


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_markstein_division(dtype):
    """div_by (shared reciprocal + Markstein correction, common.cuh) equals IEEE division bit for bit."""
    rng = np.random.default_rng(17)
    m = 4_000_000
    lo, hi = (-300, 300) if dtype == np.float64 else (-35, 35)
    a = (rng.standard_normal(m) * 10.0 ** rng.uniform(lo, hi, m)).astype(dtype)
    b = (rng.standard_normal(m) * 10.0 ** rng.uniform(lo, hi, m)).astype(dtype)
    fi = np.finfo(dtype)
    edge = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, fi.tiny, fi.tiny / 4, fi.max, -fi.max, 1.0, -1.0,
                     2.0, 0.5, 3.0, 1.0 - fi.eps / 2, 1.0 + fi.eps, fi.smallest_subnormal], dtype)
    ea, eb = np.meshgrid(edge, edge)
    ones = np.full(m // 4, 1.0, dtype) + rng.integers(0, 1 << 20, m // 4).astype(dtype) * fi.eps  # near-1 divisors
    # signed zeros over divisors of every magnitude, subnormals included (the rows that
    # pad a matrix up to its kernel's tile divide zeros at every pivot step)
    zs = np.where(rng.random(m // 4) < 0.5, 0.0, -0.0).astype(dtype)
    zd = (rng.standard_normal(m // 4) * 10.0 ** rng.uniform(lo, hi, m // 4)).astype(dtype)
    zd[::7] = (rng.standard_normal(zd[::7].size) * fi.smallest_subnormal * 1000).astype(dtype)
    a = np.concatenate([a, ea.ravel(), rng.standard_normal(m // 4).astype(dtype), zs])
    b = np.concatenate([b, eb.ravel(), ones, zd])
    ta, tb = dev(a), dev(b)
    fast, ieee = torch.empty_like(ta), torch.empty_like(ta)
    name = "tsdx_internal_div_check_" + capi.sfx(np.dtype(dtype))
    capi.check(getattr(capi.lib(), name)(capi.ptr(ta), capi.ptr(tb), capi.ptr(fast), capi.ptr(ieee), a.size,
                                        capi.stream_ptr()))
    f, e = host(fast), host(ieee)
    iv = np.uint64 if dtype == np.float64 else np.uint32
    same = (f.view(iv) == e.view(iv)) | (np.isnan(f) & np.isnan(e))
    assert same.all(), (a[~same][:5], b[~same][:5])
