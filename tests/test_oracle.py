"""Pins the CPU oracle: against the golden vectors the reference itself produced
(tests/golden/make_golden.py) and, where the compiled reference is present
(oracle/_ref), bit-for-bit against the reference on fresh inputs."""
import numpy as np
import pytest

from conftest import load_pkg

M = load_pkg("matrices")


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    iv = np.uint64 if a.dtype == np.float64 else np.uint32
    return np.array_equal(a.view(iv), b.view(iv))


def test_oracle_matches_golden_factors(oracle, golden):
    keys = [k[:-4] for k in golden.files if k.endswith("_gen")]
    assert len(keys) >= 18
    for k in keys:
        LU, piv, info = oracle.lu(golden[k + "_gen"], "auto")
        assert bits_equal(LU, golden[k + "_LU"]), k
        np.testing.assert_array_equal(piv, golden[k + "_piv"])
        np.testing.assert_array_equal(info, golden[k + "_luinfo"])
        L, cinfo = oracle.cholesky(golden[k + "_spd"], "auto")
        assert bits_equal(L, golden[k + "_L"]), k
        np.testing.assert_array_equal(cinfo, golden[k + "_info"])
        Ls, _ = oracle.cholesky(golden[k + "_spd"], "scalar")
        assert bits_equal(Ls, golden[k + "_Lscalar"]), k
        assert bits_equal(oracle.cholesky_solve(golden[k + "_L"], golden[k + "_B"]), golden[k + "_Xchol"]), k
        assert bits_equal(oracle.lu_solve(golden[k + "_LU"], golden[k + "_piv"], golden[k + "_B"]), golden[k + "_Xlu"]), k


def test_oracle_known_answers(oracle, golden):
    # tests/cpp/test_solvers.cpp:143-155: [[0,1],[1,0]] swaps rows
    for be in ("naive", "scalar", "simd", "auto"):
        LU, piv, info = oracle.lu(golden["kat_pivot2"], be)
        assert list(piv[0]) == [1, 1] and info[0] == 0 and LU[0, 0, 0] == 1 and LU[0, 1, 1] == 1
    _, info = oracle.cholesky(golden["kat_nonspd"], "auto")
    np.testing.assert_array_equal(info, golden["kat_nonspd_info"])
    assert info[3] > 0 and info[9] == 1 and (np.delete(info, [3, 9]) == 0).all()
    _, piv, info = oracle.lu(golden["kat_singular"], "auto")
    np.testing.assert_array_equal(info, golden["kat_singular_info"])
    assert info[6] == 1 and info[4] > 0
    # tests/cpp/test_precision.cpp:10-30
    xs = golden["round_x"]
    for x, h, b in zip(xs, golden["round_fp16"], golden["round_bf16"]):
        assert np.float32(oracle.round_fp16(x)).tobytes() == np.float32(h).tobytes() or (np.isnan(h) and np.isnan(oracle.round_fp16(x)))
        assert np.float32(oracle.round_bf16(x)).tobytes() == np.float32(b).tobytes()
    assert oracle.round_fp16(1.0 + 1.0 / 2048) == 1.0
    assert np.isinf(oracle.round_fp16(65520.0))
    assert oracle.round_fp16(6.0e-8) == 5.9604644775390625e-08


def test_oracle_metrics(oracle, golden):
    A, b, x = golden["metric_A"], golden["metric_b"], golden["metric_x"]
    LU, piv, _ = oracle.lu(A, "auto")
    assert bits_equal(oracle.lu_backward_error(A, LU, piv), golden["metric_lu_bwd"])
    assert bits_equal(oracle.solve_backward_error(A, x, b), golden["metric_solve_bwd"])
    assert bits_equal(oracle.solve_forward_error(A, x, b), golden["metric_solve_fwd"])
    assert bits_equal(oracle.reference_solve(A, b), golden["metric_xref"])
    S = golden["metric_S"]
    L, _ = oracle.cholesky(S, "auto")
    assert bits_equal(oracle.chol_backward_error(S, L), golden["metric_chol_bwd"])


@pytest.mark.parametrize("n", [1, 2, 3, 7, 16, 17, 24, 25, 31, 33, 50, 64])
def test_oracle_backward_error_bounds(oracle, n):
    """The reference's accuracy contract (tests/cpp/test_solvers.cpp:46-70, :111-135)."""
    rng = np.random.default_rng(100 + n)
    Mx = rng.standard_normal((19, n, n))
    S = Mx @ Mx.transpose(0, 2, 1) + n * np.eye(n)
    for be in ("naive", "scalar", "simd", "auto"):
        L, info = oracle.cholesky(S, be)
        assert (info == 0).all()
        assert oracle.chol_backward_error(S, L).max() < 4 * 2.0 ** -53 * n
        G = rng.standard_normal((19, n, n))
        LU, piv, info = oracle.lu(G, be)
        assert (info == 0).all()
        assert oracle.lu_backward_error(G, LU, piv).max() < 8 * 2.0 ** -53 * n


def test_oracle_emulated_precisions(oracle):
    rng = np.random.default_rng(3)
    for prec, u in (("fp16", 2.0 ** -11), ("bf16", 2.0 ** -8)):
        A = oracle.round_to(M.spd(rng, 20, 16, 10.0), prec)
        L, info = oracle.emu_cholesky(prec, A)
        assert (info == 0).all()
        assert (oracle.round_to(L, prec) == L).all()
        err = oracle.chol_backward_error(A, L)
        assert err.max() < 20 * u * 16 and err.max() > 2.0 ** -24


ref = pytest.importorskip("oracle.oracle")


@pytest.mark.skipif(not ref.ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_bitwise_against_compiled_reference(oracle, dtype):
    R = ref.Oracle("reference")
    rng = np.random.default_rng(11)
    for n in (1, 2, 5, 16, 17, 24, 25, 32, 33, 64):
        G = rng.standard_normal((9, n, n)).astype(dtype)
        if n > 2:
            G[2, :, 1] = 0
            G[4] = rng.integers(-2, 3, (n, n))
        S = (G @ G.transpose(0, 2, 1) + n * np.eye(n)).astype(dtype)
        for be in ("naive", "scalar", "simd", "auto"):
            a1, p1, i1 = oracle.lu(G, be)
            a2, p2, i2 = R.lu(G, be)
            assert bits_equal(a1, a2) and np.array_equal(p1, p2) and np.array_equal(i1, i2), (n, be)
            l1, j1 = oracle.cholesky(S, be)
            l2, j2 = R.cholesky(S, be)
            assert bits_equal(l1, l2) and np.array_equal(j1, j2), (n, be)
