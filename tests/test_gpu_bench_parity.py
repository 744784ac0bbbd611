"""Oracle parity on the exact inputs the benchmark times.

bench.py's dense workloads are built by its own make_inputs (kappa log-uniform per
matrix, 5% of the LU matrices with one zeroed column, the benchmark's seed for rank
0) and go through the C-ABI at their full batch. A seeded sample of 4,096 matrices,
every matrix with info > 0 and every matrix with an exactly zero column are
compared with the oracle (the C restatement of kernels.hpp, pinned bit for bit to
the reference library): factors bit for bit, pivots and info exactly, solutions
within the backward-error bound c*n*u (c = 8, the reference tests' factor
tolerance, tests/cpp/test_solvers.cpp:58, :123).

The uneven stream is checked against the oracle directly (not against the dense
kernels): a 16,384-matrix slice built like the benchmark's stream, every matrix's
factor, pivots and info compared per (kind, n, nrhs) group."""
import importlib.util

import numpy as np
import pytest

from conftest import ROOT, load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

capi = load_pkg("capi")
stream = load_pkg("stream")

SAMPLE = 4096
U = {np.float32: 2.0 ** -24, np.float64: 2.0 ** -53}
C_BWD = 8.0


def _bench():
    spec = importlib.util.spec_from_file_location("bench_for_parity", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


bench = _bench()


def bits_equal(a, b):
    iv = np.uint64 if a.dtype == np.float64 else np.uint32
    return np.array_equal(np.ascontiguousarray(a).view(iv), np.ascontiguousarray(b).view(iv))


def solve_bwd(A, X, B):
    A, X, B = (v.astype(np.float64) for v in (A, X, B))
    R = B - A @ X
    den = np.linalg.norm(A, axis=(1, 2))[:, None] * np.linalg.norm(X, axis=1) + np.linalg.norm(B, axis=1)
    return np.linalg.norm(R, axis=1) / den


def checked_indices(A, info, batch, seed):
    """The sample, every info > 0 and every matrix with an exactly zero column."""
    rng = np.random.default_rng(seed)
    zero_col = (A == 0).all(axis=1).any(axis=1)
    return np.union1d(np.union1d(rng.choice(batch, min(SAMPLE, batch), replace=False), np.nonzero(info > 0)[0]),
                      np.nonzero(zero_col)[0])


@pytest.mark.parametrize("name", ["gesv_f64_n64", "gesv_f32_n32", "gesv_f64_n32", "gesv_f32_n64", "posv_f64_n16"])
def test_bench_inputs_match_oracle(oracle, name):
    kind, n, batch, nrhs, dt, klo, khi, zf = bench.WORKLOADS[name]
    dtype = torch.float64 if dt == "f64" else torch.float32
    A, B = bench.make_inputs(torch, kind, n, batch, nrhs, dtype, klo, khi, zf, 1234, "cuda")
    A0, B0 = A.cpu().numpy(), B.cpu().numpy()
    info = torch.full((batch,), -7, dtype=torch.int32, device="cuda")
    if kind == "gesv":
        piv = torch.zeros(batch, n, dtype=torch.int32, device="cuda")
        capi.gesv(A, B, piv, info)
    else:
        capi.posv(A, B, info)
    torch.cuda.synchronize()
    F, X, I = A.cpu().numpy(), B.cpu().numpy(), info.cpu().numpy()
    idx = checked_indices(A0, I, batch, 5)
    if kind == "gesv":
        P = piv.cpu().numpy()
        Fo, Po, Io = oracle.lu(A0[idx], "scalar")
        np.testing.assert_array_equal(P[idx], Po)
        # the planted zero columns (5% of the LU matrices) all end with info > 0
        assert (I > 0).sum() >= 0.04 * batch
    else:
        Fo, Io = oracle.cholesky(A0[idx], "simd")
    np.testing.assert_array_equal(I[idx], Io)
    assert bits_equal(F[idx], Fo)
    ok = Io == 0
    bwd = solve_bwd(A0[idx][ok], X[idx][ok], B0[idx][ok])
    assert bwd.max() <= C_BWD * n * U[A0.dtype.type], bwd.max()


def test_bench_stream_slice_matches_oracle(oracle):
    count = 16384
    n, nrhs, kind, A, B = bench.stream_inputs(count, 0, "cuda")
    A0, B0 = A.cpu().numpy(), B.cpu().numpy()
    aoff, boff, poff, na, nb, npv = stream.layout(n, nrhs)
    plan = stream.StreamPlan(n, nrhs, kind, torch.float32, device="cuda")
    plan.capture()  # the capture runs one warm-up solve on the plan's buffers: load after it
    plan.load(A, B)
    plan.run()
    torch.cuda.synchronize()
    F, X = plan.A.cpu().numpy(), plan.B.cpu().numpy()
    P, I = plan.piv.cpu().numpy(), plan.info.cpu().numpy()
    ao, bo, po = aoff.numpy(), boff.numpy(), poff.numpy()
    checked = 0
    for kk in (0, 1):
        for nn in np.unique(n):
            idx = np.nonzero((kind == kk) & (n == nn))[0]
            for r in np.unique(nrhs[idx]):
                g = idx[nrhs[idx] == r]
                a = np.stack([A0[ao[i]:ao[i] + nn * nn].reshape(nn, nn) for i in g])
                b = np.stack([B0[bo[i]:bo[i] + nn * r].reshape(nn, r) for i in g])
                f = np.stack([F[ao[i]:ao[i] + nn * nn].reshape(nn, nn) for i in g])
                x = np.stack([X[bo[i]:bo[i] + nn * r].reshape(nn, r) for i in g])
                if kk == 1:
                    fo, pvo, io = oracle.lu(a, "scalar")
                    p = np.stack([P[po[i]:po[i] + nn] for i in g])
                    np.testing.assert_array_equal(p, pvo)
                else:
                    fo, io = oracle.cholesky(a, "simd")
                np.testing.assert_array_equal(I[g], io)
                assert bits_equal(f, fo), (kk, nn, r)
                ok = io == 0
                if ok.any():
                    bwd = solve_bwd(a[ok], x[ok], b[ok])
                    assert bwd.max() <= C_BWD * nn * U[np.float32], (kk, nn, r, bwd.max())
                checked += len(g)
    assert checked == count
