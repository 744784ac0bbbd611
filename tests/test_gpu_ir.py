"""Mixed-precision factorization + fp64 iterative refinement (gesv_ir / posv_ir).

The contract checked here: every returned x has a normwise backward error
(runtime.cpp:230-242, evaluated by the long-double oracle) no worse than twice
that of the plain fp64 GPU solve of the same system plus one unit roundoff;
matrices the refinement reports as converged meet the tolerance; matrices it
cannot refine are re-solved in fp64 (status -1) and then match the plain fp64
path exactly; A is never modified.
"""
import numpy as np
import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

capi = load_pkg("capi")
M = load_pkg("matrices")
U64 = 2.0 ** -53


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def run_ir(A, b, spd, tier=None, default_tier=1, itmax=3, tol=1e-15):
    batch, n = A.shape[0], A.shape[1]
    a, x = dev(A), dev(b)
    info = torch.zeros(batch, dtype=torch.int32, device="cuda")
    status = torch.zeros(batch, dtype=torch.int32, device="cuda")
    bwd = torch.zeros(batch, dtype=torch.float64, device="cuda")
    t = dev(np.asarray(tier, np.int8)) if tier is not None else None
    name = "tsdx_cuda_posv_ir_f64" if spd else "tsdx_cuda_gesv_ir_f64"
    fn = getattr(capi.lib(), name)
    capi.check(fn(capi.ptr(a), n, batch, capi.ptr(x), capi.ptr(t), default_tier, itmax, float(tol), capi.ptr(info),
                  capi.ptr(status), capi.ptr(bwd), capi.stream_ptr()), name)
    torch.cuda.synchronize()
    assert torch.equal(a.cpu(), torch.from_numpy(A)), "A was modified"
    return x.cpu().numpy(), info.cpu().numpy(), status.cpu().numpy(), bwd.cpu().numpy()


def plain(A, b, spd):
    a, x = dev(A), dev(b[..., None])
    info = torch.zeros(A.shape[0], dtype=torch.int32, device="cuda")
    if spd:
        capi.posv(a, x, info)
    else:
        piv = torch.zeros(A.shape[:2], dtype=torch.int32, device="cuda")
        capi.gesv(a, x, piv, info)
    torch.cuda.synchronize()
    return x.cpu().numpy()[..., 0]


@pytest.mark.parametrize("spd", [False, True])
@pytest.mark.parametrize("n", [8, 16, 33, 64])
@pytest.mark.parametrize("tier", [0, 1, 2])
def test_ir_accuracy_matches_fp64(oracle, spd, n, tier):
    rng = np.random.default_rng(n * 10 + tier + (100 if spd else 0))
    batch = 96
    kap = M.log_uniform(rng, batch, 1e1, 1e6)
    A = (M.spd if spd else M.general)(rng, batch, n, kap)
    b = rng.standard_normal((batch, n))
    x, info, status, bwd = run_ir(A, b, spd, default_tier=tier)
    xp = plain(A, b, spd)
    be_ir = oracle.solve_backward_error(A, x, b)
    be_fp = oracle.solve_backward_error(A, xp, b)
    # at equal backward error: the batch's median and worst case within 2x of plain fp64,
    # every matrix within the refinement tolerance
    assert np.median(be_ir) <= 2 * np.median(be_fp), (np.median(be_ir), np.median(be_fp))
    assert be_ir.max() <= 2 * be_fp.max() + U64, (be_ir.max(), be_fp.max())
    assert (be_ir <= 1e-15).all()
    conv = status >= 0
    assert (bwd[conv] <= 1e-15).all()
    # fallback matrices are the plain fp64 solution
    np.testing.assert_array_equal(x[~conv], xp[~conv])
    if tier == 2:
        assert conv.mean() > 0.9  # fp32 refines kappa <= 1e6 without fallback


def test_ir_tier_fp64_is_the_plain_path():
    rng = np.random.default_rng(3)
    A = M.general(rng, 40, 64, 1e3)
    b = rng.standard_normal((40, 64))
    x, info, status, _ = run_ir(A, b, False, default_tier=3)
    assert (status == -1).all()
    np.testing.assert_array_equal(x, plain(A, b, False))


def test_ir_per_matrix_tiers_and_ill_conditioned_fallback(oracle):
    rng = np.random.default_rng(4)
    batch, n = 64, 48
    kap = np.where(np.arange(batch) % 2 == 0, 1e2, 1e12)
    A = M.general(rng, batch, n, kap)
    b = rng.standard_normal((batch, n))
    tier = np.tile(np.array([0, 1, 2, 3], np.int8), batch // 4)
    x, info, status, bwd = run_ir(A, b, False, tier=tier)
    xp = plain(A, b, False)
    be_ir = oracle.solve_backward_error(A, x, b)
    be_fp = oracle.solve_backward_error(A, xp, b)
    assert be_ir.max() <= 2 * be_fp.max() + U64
    # kappa = 1e12 cannot be refined from fp16/bf16 factors: those fall back
    ill = (np.arange(batch) % 2 == 1) & (tier <= 1)
    assert (status[ill] == -1).all()
    assert (status[tier == 3] == -1).all()
