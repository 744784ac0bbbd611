"""Emulated fp16 / bf16 (per-operation rounding, precision.hpp:41-97) on the GPU:
bit-identical to the CPU path of the drop-in and to the pinned checker (NaN where
they have NaN), for the factorizations and the solves, float64 and float32
storage, including failures."""
import numpy as np
import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

tsdx = load_pkg()
M = load_pkg("matrices")


def same(a, b):
    """Bit-identical, NaN where the other has NaN (payloads are not compared: x86
    arithmetic carries an input NaN's payload through, the GPU makes a canonical one)."""
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    iv = np.uint64 if a.dtype == np.float64 else (np.uint32 if a.dtype == np.float32 else np.uint16)
    return bool(((a.view(iv) == b.view(iv)) | (np.isnan(a) & np.isnan(b))).all())


@pytest.mark.parametrize("prec", ["fp16", "bf16"])
@pytest.mark.parametrize("n", [1, 2, 5, 16, 33, 64])
def test_emulated_gpu_equals_cpu(oracle, prec, n):
    r = np.random.default_rng(n)
    S = M.spd(r, 7, n, 30.0)
    G = r.standard_normal((7, n, n))
    if n > 3:
        S[2, 1, 1] = -1.0       # not positive definite: early exit keeps the upper triangle
        G[3, :, 2] = 0.0        # a zero pivot column
        G[4, 0, 0] = np.nan
    B = r.standard_normal((7, n, 3))
    L, info = tsdx.cholesky(S, precision=prec, backend="cuda")
    Lc, infoc = tsdx.cholesky(S, precision=prec, backend="scalar")
    assert same(L, Lc) and np.array_equal(info, infoc)
    Lo, infoo = oracle.emu_cholesky(prec, S)
    assert same(L, Lo) and np.array_equal(info, infoo)
    LU, piv, info = tsdx.lu(G, precision=prec, backend="cuda")
    LUc, pivc, infoc = tsdx.lu(G, precision=prec, backend="scalar")
    assert same(LU, LUc) and np.array_equal(piv, pivc) and np.array_equal(info, infoc)
    ok = infoc == 0
    X = tsdx.lu_solve(LUc, pivc, B, precision=prec, backend="cuda")
    Xc = tsdx.lu_solve(LUc, pivc, B, precision=prec, backend="scalar")
    assert same(X[ok], Xc[ok])
    Sg = M.spd(r, 7, n, 30.0)
    Lg, _ = tsdx.cholesky(Sg, precision=prec, backend="scalar")
    assert same(tsdx.cholesky_solve(Lg, B, precision=prec, backend="cuda"),
                tsdx.cholesky_solve(Lg, B, precision=prec, backend="scalar"))


def test_emulated_float32_and_float16_storage():
    r = np.random.default_rng(3)
    S = M.spd(r, 5, 12, 10.0).astype(np.float32)
    L, info = tsdx.cholesky(S, precision="fp16", backend="cuda")
    Lc, infoc = tsdx.cholesky(S, precision="fp16", backend="auto")
    assert L.dtype == np.float32 and same(L, Lc) and np.array_equal(info, infoc)
    H = S.astype(np.float16)
    L, info = tsdx.cholesky(H, backend="cuda")
    Lc, _ = tsdx.cholesky(H, backend="auto")
    assert L.dtype == np.float16 and same(L, Lc)
