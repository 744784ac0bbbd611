"""The learned precision-tier selector on the GPU: features, forward pass,
gradients and Adam step against the float64 CPU checker; training on labels made
by the refinement kernel itself; and the A/B comparison with the method without
the network (every matrix first tries the cheapest tier and falls back to fp64 on
a miss)."""
import numpy as np
import pytest

from conftest import load_pkg
from oracle import selector_ref as R

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

sel = load_pkg("selector")
device = load_pkg("device")
M = load_pkg("matrices")
U64 = 2.0 ** -53


def stack(seed, batch, n, spd, klo=1.0, khi=1e14):
    rng = np.random.default_rng(seed)
    kap = M.log_uniform(rng, batch, klo, khi)
    A = (M.spd if spd else M.general)(rng, batch, n, kap)
    b = rng.standard_normal((batch, n))
    return A, b


@pytest.mark.parametrize("n", [1, 2, 7, 33, 64])
@pytest.mark.parametrize("spd", [False, True])
def test_features_match_oracle(n, spd):
    A, _ = stack(n, 50, n, spd, 1.0, 1e10)
    if n > 3:
        A[3, 1, :] = 0.0  # zero row: clipped ratios
        A[4] = np.diag(np.arange(1.0, n + 1))
    f = sel.features(torch.from_numpy(A).cuda(), 0 if spd else 1).cpu().numpy()
    fo = R.features(A, 0 if spd else 1)
    np.testing.assert_allclose(f, fo, rtol=1e-5, atol=2e-5)
    kind = torch.tensor(np.arange(50) % 2, dtype=torch.int8, device="cuda")
    f2 = sel.features(torch.from_numpy(A).cuda(), kind).cpu().numpy()
    assert np.array_equal(f2[:, 1], np.arange(50) % 2)


def test_forward_grad_adam_match_oracle():
    rng = np.random.default_rng(7)
    s = sel.Selector(seed=3)
    X = rng.normal(0, 3, (300, 24)).astype(np.float32)
    y = rng.integers(0, 4, 300).astype(np.int8)
    Xd = torch.from_numpy(X).cuda()
    s.fit_normalizer(Xd)
    P = s.params.cpu().numpy().astype(np.float64)
    norm = s.norm.cpu().numpy().astype(np.float64)
    logits, tier = s.forward(Xd)
    lo, _ = R.forward(P, norm, X)
    np.testing.assert_allclose(logits.cpu().numpy(), lo, rtol=1e-4, atol=1e-4)
    top = np.sort(lo, 1)
    clear = top[:, -1] - top[:, -2] > 1e-3
    assert np.array_equal(tier.cpu().numpy()[clear], lo.argmax(1)[clear])
    cw = np.array([2.0, 1.0, 0.5, 1.0])
    g, loss = s.loss_grad(Xd, torch.from_numpy(y).cuda(), cw)
    lref, gref = R.loss_and_grad(P, norm, X, y, cw)
    assert abs(loss.item() - lref) <= 1e-5 * abs(lref)
    g = g.cpu().numpy()
    assert np.abs(g - gref).max() <= 1e-4 * np.abs(gref).max() + 1e-7
    m0, v0 = s.m.cpu().numpy(), s.v.cpu().numpy()
    s.adam_step(torch.from_numpy(g).cuda(), lr=1e-2)
    P1, _, _ = R.adam(P, g.astype(np.float64), m0, v0, 1, 1e-2)
    np.testing.assert_allclose(s.params.cpu().numpy(), P1, atol=1e-6)


def make_set(seed, per, sizes=(16, 32, 48, 64)):
    """Features, labels (from the refinement kernel) and the stacks, per (n, kind)."""
    groups = []
    for i, n in enumerate(sizes):
        for spd in (False, True):
            A, b = stack(seed * 100 + i * 2 + spd, per, n, spd)
            Ad, bd = torch.from_numpy(A).cuda(), torch.from_numpy(b).cuda()
            groups.append((n, spd, A, b, sel.features(Ad, 0 if spd else 1), sel.label(Ad, bd, spd)))
    X = torch.cat([g[4] for g in groups])
    y = torch.cat([g[5] for g in groups])
    return groups, X, y


def test_training_learns_and_beats_the_method_without_it(oracle):
    _, X, y = make_set(1, 1500)
    counts = torch.bincount(y.long(), minlength=4).cpu().numpy()
    assert counts[3] > 0 and counts[:3].sum() > 0, counts
    s = sel.Selector(seed=0)
    hist = s.fit(X, y, epochs=30, batch_size=1024, lr=3e-3)
    assert hist[-1] < 0.7 * hist[0], hist
    groups, Xe, ye = make_set(2, 400)
    pred = s.predict(Xe)
    acc = (pred == ye).float().mean().item()
    majority = torch.bincount(ye.long(), minlength=4).max().item() / len(ye)
    assert acc > majority + 0.02, (acc, majority)
    # A/B on held-out matrices: fp64 fallbacks (a low-precision attempt that missed)
    # with the network vs trying fp16 first for every matrix
    miss_sel = miss_fixed = lowprec = 0
    for n, spd, A, b, F, _ in groups:
        Ad = torch.from_numpy(A).cuda()
        x = torch.from_numpy(b).cuda()
        info, status, bwd, tier = s.solve(Ad, x, spd)
        st, t = status.cpu().numpy(), tier.cpu().numpy()
        miss_sel += int(((t < 3) & (st < 0)).sum())
        lowprec += int((st >= 0).sum())
        xf = torch.from_numpy(b).cuda()
        _, st_fixed, _ = device.ir(Ad, xf, spd, default_tier=0)
        miss_fixed += int((st_fixed < 0).sum().item())
        # accuracy: the selector's solutions stay within 2x the plain fp64 backward error
        xp = torch.from_numpy(b).cuda().unsqueeze(-1).contiguous()
        a2 = Ad.clone()
        (device.posv(a2, xp) if spd else device.gesv(a2, xp))
        be = oracle.solve_backward_error(A, x.cpu().numpy(), b)
        bp = oracle.solve_backward_error(A, xp.cpu().numpy()[..., 0], b)
        assert be.max() <= 2 * bp.max() + U64
    print(f"selector: {miss_sel} misses, {lowprec} refined; fp16-first: {miss_fixed} misses")
    assert miss_sel < 0.5 * miss_fixed
    assert lowprec > 0


@pytest.mark.parametrize("shipped", [True, False])
def test_solve_host_matches_device_solve(shipped):
    """Selector.solve_host (host buffers, chunks pipelined over 3 streams, several parts)
    returns x, info, status and tier bit-identical to the device solve of each whole part.
    shipped: the committed weights and cost table (every order routed to fp64); else an
    untrained network without costs, so predicted tiers, refinement and fallbacks all run."""
    import pathlib
    s = (sel.Selector.load(str(pathlib.Path(sel.__file__).parent / "selector_weights.npz")) if shipped
         else sel.Selector(seed=3))
    parts, ref = [], []
    for i, (n, spd, batch) in enumerate([(64, False, 40), (17, True, 300), (5, False, 7), (64, True, 0)]):
        A, b = stack(900 + i, max(batch, 1), n, spd, 1.0, 1e12)
        A, b = A[:batch], b[:batch]
        Ad, bd = torch.from_numpy(A).cuda(), torch.from_numpy(b).cuda()
        if batch:
            info, status, _, tier = s.solve(Ad, bd, spd)
        else:
            info = status = torch.zeros(0, dtype=torch.int32)
            tier = torch.zeros(0, dtype=torch.int8)
        ref.append((bd.cpu(), info.cpu(), status.cpu(), tier.cpu()))
        hA = torch.from_numpy(np.ascontiguousarray(A))
        parts.append((hA.pin_memory() if i % 2 == 0 else hA, torch.from_numpy(np.ascontiguousarray(b)), spd))
    outs = s.solve_host(parts, chunk_bytes=64 * 64 * 8 * 3)  # 3 matrices of order 64 per chunk
    for (_, hb, _), (info, status, tier), (x, i0, s0, t0) in zip(parts, outs, ref):
        assert torch.equal(hb.view(torch.int64), x.view(torch.int64))
        assert torch.equal(info, i0) and torch.equal(status, s0) and torch.equal(tier, t0)
    if not shipped:
        assert int((ref[0][3] < 3).sum()) > 0  # lower tiers did run
