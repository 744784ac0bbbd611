"""The uneven stream (one call over mixed n, Cholesky and LU mixed, 0..8 RHS): every
factor, pivot, info and solution bit-identical to the dense posv/gesv kernels of the
same matrix, through the C-ABI directly, the autotuned CUDA-graph plan and the
NumPy-facing solve_stream."""
import numpy as np
import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

tsdx = load_pkg()
matrices = load_pkg("matrices")
device = load_pkg("device")
stream = load_pkg("stream")


def bits_equal(a, b):
    a, b = a.contiguous(), b.contiguous()
    iv = torch.int64 if a.dtype == torch.float64 else torch.int32
    return torch.equal(a.view(iv), b.view(iv))


def make_stream(seed, count, dtype, nmax=64, rhs=(0, 1, 2, 3, 4, 5, 8), zero_frac=0.05):
    """Packed host tensors for a random mixed stream (SPD for Cholesky, general for LU)."""
    r = np.random.default_rng(seed)
    n = r.integers(1, nmax + 1, count).astype(np.int32)
    kind = r.integers(0, 2, count).astype(np.int8)
    nrhs = r.choice(rhs, count).astype(np.int32)
    mats, bs = [], []
    for i in range(count):
        k = matrices.log_uniform(r, 1, 1e1, 1e8)
        a = (matrices.spd if kind[i] == 0 else matrices.general)(r, 1, int(n[i]), k)[0]
        if kind[i] == 1 and n[i] > 2 and r.random() < zero_frac:
            a[:, r.integers(n[i])] = 0
        if kind[i] == 0 and n[i] > 2 and r.random() < zero_frac:
            a[n[i] // 2, n[i] // 2] = -1.0
        mats.append(a.astype(dtype))
        bs.append(r.standard_normal((int(n[i]), int(nrhs[i]))).astype(dtype))
    A = torch.from_numpy(np.concatenate([m.ravel() for m in mats]))
    B = torch.from_numpy(np.concatenate([b.ravel() for b in bs] + [np.zeros(1, dtype)]))
    return n, nrhs, kind, mats, bs, A, B


def dense_reference(n, nrhs, kind, mats, bs, dtype):
    """Per (kind, n, nrhs) group: the dense device posv/gesv kernels."""
    out = {}
    groups = {}
    for i in range(len(n)):
        groups.setdefault((int(kind[i]), int(n[i]), int(nrhs[i])), []).append(i)
    for (k, nn, rr), idx in groups.items():
        A = torch.from_numpy(np.stack([mats[i] for i in idx])).cuda()
        B = torch.from_numpy(np.stack([bs[i] for i in idx]).reshape(len(idx), nn, rr)).cuda()
        if rr == 0:
            B = torch.zeros(len(idx), nn, 1, dtype=A.dtype, device="cuda")
        if k == 0:
            info = device.posv(A, B)
            piv = None
        else:
            piv, info = device.gesv(A, B)
        for j, i in enumerate(idx):
            out[i] = (A[j].cpu(), B[j, :, :rr].cpu(), None if piv is None else piv[j].cpu(), int(info[j]))
    return out


def check_against_dense(n, nrhs, kind, ref, A, B, piv, info, wf=True):
    aoff, boff, poff, *_ = stream.layout(torch.from_numpy(n), torch.from_numpy(nrhs))
    A, B, piv, info = A.cpu(), B.cpu(), piv.cpu(), info.cpu()
    bad = []
    for i in range(len(n)):
        nn, rr = int(n[i]), int(nrhs[i])
        F, X, P, inf = ref[i]
        ok = int(info[i]) == inf
        if wf:
            ok &= bits_equal(A[aoff[i]:aoff[i] + nn * nn].view(nn, nn), F)
            if kind[i]:
                ok &= torch.equal(piv[poff[i]:poff[i] + nn], P)
        if rr and inf == 0:
            ok &= bits_equal(B[boff[i]:boff[i] + nn * rr].view(nn, rr), X)
        if not ok:
            bad.append((i, int(kind[i]), nn, rr))
    assert not bad, f"{len(bad)} mismatches, first {bad[:5]}"


def run_direct(n, nrhs, kind, A, B, wf=True, sched=0, scratch=True):
    aoff, boff, poff, na, nb, npv = stream.layout(torch.from_numpy(n), torch.from_numpy(nrhs))
    d = "cuda"
    Ad, Bd = A.to(d), B.to(d)
    piv = torch.zeros(max(npv, 1), dtype=torch.int32, device=d)
    info = torch.full((len(n),), 77, dtype=torch.int32, device=d)
    sc = torch.empty(stream.scratch_bytes(len(n)), dtype=torch.uint8, device=d) if scratch else None
    stream.solve(Ad, aoff.to(d), Bd, boff.to(d), piv, poff.to(d), info, torch.from_numpy(n).to(d),
                 torch.from_numpy(nrhs).to(d), torch.from_numpy(kind).to(d), wf, sched, sc)
    torch.cuda.synchronize()
    return Ad, Bd, piv, info


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("sched", [0, 15, 5])
def test_stream_bit_identical_to_dense(dtype, sched):
    n, nrhs, kind, mats, bs, A, B = make_stream(11 + sched, 1500, dtype)
    ref = dense_reference(n, nrhs, kind, mats, bs, dtype)
    Ad, Bd, piv, info = run_direct(n, nrhs, kind, A, B, sched=sched, scratch=sched == 0)
    assert (info.cpu() != 77).all()
    check_against_dense(n, nrhs, kind, ref, Ad, Bd, piv, info)


def test_stream_solution_only_and_small_sizes():
    # n <= 16 only: the packed (several matrices per warp) units dominate; x-only mode
    n, nrhs, kind, mats, bs, A, B = make_stream(5, 3000, np.float32, nmax=16)
    ref = dense_reference(n, nrhs, kind, mats, bs, np.float32)
    Ad, Bd, piv, info = run_direct(n, nrhs, kind, A, B, wf=False, sched=1)
    check_against_dense(n, nrhs, kind, ref, Ad, Bd, piv, info, wf=False)
    assert torch.equal(Ad.cpu(), A)  # A untouched without write_factors


def test_stream_invalid_entries_flagged():
    n = np.array([3, 0, 65, 4, 5, -2], np.int32)
    nrhs = np.array([1, 1, 1, 9, 2, 1], np.int32)
    kind = np.array([0, 1, 0, 1, 1, 0], np.int8)
    r = np.random.default_rng(0)
    mats = [matrices.spd(r, 1, 3, 10.0)[0], np.zeros((0, 0)), np.zeros((0, 0)), np.eye(4), np.eye(5) * 2,
            np.zeros((0, 0))]
    sz = [max(int(k), 0) for k in n]
    A = torch.zeros(sum(s * s for s in sz), dtype=torch.float64)
    A[:9] = torch.from_numpy(mats[0].ravel())
    o = 9 + 0 + 65 * 65
    A[o:o + 16] = torch.eye(4, dtype=torch.float64).ravel()
    A[o + 16:o + 41] = 2 * torch.eye(5, dtype=torch.float64).ravel()
    # layout of negative n is clamped by the caller; build offsets by hand
    aoff = torch.tensor([0, 9, 9, o, o + 16, o + 41])
    boff = torch.tensor([0, 3, 3, 68, 104, 114])
    poff = torch.tensor([0, 3, 3, 68, 72, 77])
    B = torch.ones(200, dtype=torch.float64)
    d = "cuda"
    Ad, Bd = A.to(d), B.to(d)
    piv = torch.zeros(100, dtype=torch.int32, device=d)
    info = torch.full((6,), 77, dtype=torch.int32, device=d)
    stream.solve(Ad, aoff.to(d), Bd, boff.to(d), piv, poff.to(d), info, torch.from_numpy(n).to(d),
                 torch.from_numpy(nrhs).to(d), torch.from_numpy(kind).to(d), True, 0, None)
    assert info.cpu().tolist() == [0, -1, -1, -1, 0, -1]
    x = Bd.cpu()[104:114].view(5, 2)
    assert torch.equal(x, torch.full((5, 2), 0.5, dtype=torch.float64))
    np.testing.assert_allclose(Bd.cpu()[:3].numpy(), np.linalg.solve(mats[0], np.ones(3)), rtol=1e-12)
    assert torch.equal(Bd.cpu()[68:104], torch.ones(36, dtype=torch.float64))  # nrhs = 9 untouched


def test_stream_empty():
    e = torch.zeros(0, device="cuda")
    z = torch.zeros(0, dtype=torch.int32, device="cuda")
    o = torch.zeros(0, dtype=torch.int64, device="cuda")
    stream.solve(torch.zeros(1, device="cuda"), o, e, o, z, o, z, z, z, torch.zeros(0, dtype=torch.int8, device="cuda"))


def test_plan_autotune_graph_replay():
    n, nrhs, kind, mats, bs, A, B = make_stream(21, 2500, np.float32, rhs=(1, 2, 4, 8))
    ref = dense_reference(n, nrhs, kind, mats, bs, np.float32)
    plan = stream.StreamPlan(n, nrhs, kind, torch.float32)
    B = B[:-1]  # drop make_stream's trailing pad element
    best = plan.tune(A, B, reps=2)
    assert 0 <= best < (1 << stream.SCHED_BITS) and len(plan.timings) >= 2
    plan.capture()
    for _ in range(2):  # replay twice on fresh inputs
        plan.load(A, B)
        plan.info.fill_(77)
        plan.run()
        torch.cuda.synchronize()
        check_against_dense(n, nrhs, kind, ref, plan.A, plan.B, plan.piv, plan.info)


def test_numpy_solve_stream():
    r = np.random.default_rng(3)
    mats = [matrices.spd(r, 1, 5, 10.0)[0], matrices.general(r, 1, 33, 1e3)[0], matrices.general(r, 1, 2, 10.0)[0]]
    rhs = [r.standard_normal(5), r.standard_normal((33, 3)), None]
    X, info, F, P = tsdx.solve_stream(mats, rhs, ["cholesky", "lu", "lu"], write_factors=True)
    assert list(info) == [0, 0, 0] and X[0].shape == (5,) and X[1].shape == (33, 3) and X[2].shape == (2, 0)
    x0, _ = tsdx.posv(mats[0], rhs[0], backend="cuda")
    x1, _ = tsdx.gesv(mats[1], rhs[1], backend="cuda")
    assert np.array_equal(X[0], x0) and np.array_equal(X[1], x1)
    LU, piv, _ = tsdx.lu(mats[1], backend="cuda")
    assert np.array_equal(F[1], LU) and np.array_equal(P[1], piv) and P[0] is None


def packed_random_stream(seed, count, dtype, nmax=64):
    """A large packed stream built per order group (SPD M M^T + n I for Cholesky,
    Gaussian for LU): no per-matrix Python work, so it can span several chunks."""
    r = np.random.default_rng(seed)
    n = r.integers(1, nmax + 1, count).astype(np.int32)
    kind = r.integers(0, 2, count).astype(np.int8)
    nrhs = r.choice([0, 1, 2, 4, 8], count).astype(np.int32)
    aoff, boff, _, na, nb, _ = stream.layout(torch.from_numpy(n), torch.from_numpy(nrhs))
    aoff, boff = aoff.numpy(), boff.numpy()
    A = np.empty(na, dtype)
    B = r.standard_normal(max(nb, 1)).astype(dtype)
    for nn in np.unique(n):
        idx = np.nonzero(n == nn)[0]
        G = r.standard_normal((idx.size, nn, nn))
        S = G @ G.transpose(0, 2, 1) + nn * np.eye(nn)
        M = np.where((kind[idx] == 0)[:, None, None], S, G).astype(dtype)
        A[aoff[idx, None] + np.arange(nn * nn)[None, :]] = M.reshape(idx.size, -1)
    return n, nrhs, kind, torch.from_numpy(A), torch.from_numpy(B)


def run_host_call(n, nrhs, kind, A, B, wf=True, sched=0, pin=False, piv_fill=0):
    _, _, _, na, nb, npv = stream.layout(torch.from_numpy(n), torch.from_numpy(nrhs))
    A, B = A.clone(), B.clone()
    piv = torch.full((max(npv, 1),), piv_fill, dtype=torch.int32)
    info = torch.full((len(n),), 77, dtype=torch.int32)
    if pin:
        A, B, piv, info = A.pin_memory(), B.pin_memory(), piv.pin_memory(), info.pin_memory()
    stream.solve_host(A, B, piv, info, torch.from_numpy(n), torch.from_numpy(nrhs), torch.from_numpy(kind), wf, sched)
    return A, B, piv, info


def check_host_equals_device(host_out, dev_out, wf):
    hA, hB, hP, hI = host_out
    dA, dB, dP, dI = (t.cpu() for t in dev_out)
    assert torch.equal(hI, dI)
    assert bits_equal(hB, dB)
    if wf:
        assert bits_equal(hA, dA) and torch.equal(hP, dP)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("wf,sched", [(True, 0), (False, 15)])
def test_stream_host_small_pageable(dtype, wf, sched):
    """Host-memory stream call (one chunk, pageable buffers) == the device stream call."""
    n, nrhs, kind, mats, bs, A, B = make_stream(41, 300, dtype)
    check_host_equals_device(run_host_call(n, nrhs, kind, A, B, wf, sched),
                             run_direct(n, nrhs, kind, A, B, wf, sched), wf)
    if wf:  # and against the dense kernels directly
        hA, hB, hP, hI = run_host_call(n, nrhs, kind, A, B, wf, sched)
        check_against_dense(n, nrhs, kind, dense_reference(n, nrhs, kind, mats, bs, dtype), hA, hB, hP, hI)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_stream_host_many_chunks_pinned(dtype):
    """A set of several 96 MB chunks from pinned memory: every matrix bit-identical to
    the single device call over the whole set (chunk boundaries and rebased offsets)."""
    count = 90_000 if dtype == np.float32 else 45_000  # about 500 MB of A: 5 or 6 chunks
    n, nrhs, kind, A, B = packed_random_stream(5, count, dtype)
    assert A.numel() * A.element_size() > 4 * (96 << 20)
    host = run_host_call(n, nrhs, kind, A, B, True, 0, pin=True, piv_fill=-7)
    dev_out = run_direct(n, nrhs, kind, A, B, True, 0)
    # Cholesky matrices get no pivots: their slots keep the caller's -7, the LU slots
    # match the device call
    _, _, poff, *_ = stream.layout(torch.from_numpy(n), torch.from_numpy(nrhs))
    chol = torch.from_numpy(np.repeat(kind == 0, n))
    assert (host[2][:chol.numel()][chol] == -7).all()
    dP = dev_out[2].cpu()
    dP[:chol.numel()][chol] = -7
    check_host_equals_device(host, (dev_out[0], dev_out[1], dP, dev_out[3]), True)
    assert (host[3] == 0).mean(dtype=torch.float64) > 0.4  # the SPD half factors (info 0)


def test_stream_host_no_rhs_no_info():
    """Factor-only use of the host-memory call: every nrhs 0 (B NULL) and no info
    buffer; factors and pivots match the device call."""
    n, nrhs, kind, A, B = packed_random_stream(9, 3000, np.float64)
    nrhs[:] = 0
    _, _, _, na, nb, npv = stream.layout(torch.from_numpy(n), torch.from_numpy(nrhs))
    assert nb == 0
    hA = A.clone()
    piv = torch.zeros(npv, dtype=torch.int32)
    stream.solve_host(hA, None, piv, None, torch.from_numpy(n), torch.from_numpy(nrhs), torch.from_numpy(kind))
    dA, _, dP, _ = run_direct(n, nrhs, kind, A, B[:1], True, 0)
    assert bits_equal(hA, dA.cpu())
    assert torch.equal(piv, dP.cpu())
