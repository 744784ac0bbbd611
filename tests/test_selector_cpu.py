"""The selector's CPU checker (oracle/selector_ref.py) pinned by exact properties,
and the selector C-ABI's argument checks (no device needed)."""
import numpy as np

from conftest import load_pkg
from oracle import selector_ref as R

capi = load_pkg("capi")


def rand_params(rng, scale=0.3):
    return rng.normal(0, scale, R.N_PARAM)


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    P = rand_params(rng)
    norm = np.concatenate([rng.normal(0, 1, 24), rng.uniform(0.5, 2, 24)])
    X = rng.normal(0, 2, (37, 24))
    y = rng.integers(0, 4, 37)
    cw = np.array([1.0, 2.0, 0.5, 1.5])
    loss, g = R.loss_and_grad(P, norm, X, y, cw)
    assert g.shape == (R.N_PARAM,)
    idx = np.concatenate([rng.choice(R.N_PARAM, 60, replace=False),
                          [R.OFF_B1, R.OFF_B2, R.OFF_B3, R.OFF_B3 + 3, R.N_PARAM - 1]])
    h = 1e-6
    for i in idx:
        e = np.zeros(R.N_PARAM)
        e[i] = h
        fd = (R.loss_and_grad(P + e, norm, X, y, cw)[0] - R.loss_and_grad(P - e, norm, X, y, cw)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])) + 1e-9, (i, fd, g[i])


def test_loss_is_weighted_mean_cross_entropy():
    rng = np.random.default_rng(1)
    P = rand_params(rng)
    norm = np.concatenate([np.zeros(24), np.ones(24)])
    X = rng.normal(size=(9, 24))
    y = rng.integers(0, 4, 9)
    logits, _ = R.forward(P, norm, X)
    p = np.exp(logits - logits.max(1, keepdims=True))
    p /= p.sum(1, keepdims=True)
    ce = -np.log(p[np.arange(9), y])
    cw = np.array([3.0, 1.0, 1.0, 0.25])
    assert np.isclose(R.loss_and_grad(P, norm, X, y, cw)[0], (cw[y] * ce).sum() / 9)


def test_features_closed_forms():
    n = 5
    A = np.diag(10.0 ** np.arange(n))[None]
    f = R.features(A, 0)[0]
    assert f[0] == n / 64 and f[1] == 0
    assert np.isclose(f[2], n - 1) and np.isclose(f[3], n - 1) and np.isclose(f[4], n - 1)
    assert f[5] == 0 and np.isclose(f[6], n - 1)
    assert f[7] == 1 and f[8] == 1 and f[9] == 1 and f[11] == 0
    assert np.isclose(f[15], np.std(np.arange(n)))
    assert f[18] == 0 and f[20] == 0 and f[22] == 0
    # a zero row: infinite ratios clip at 30, Gershgorin indicator set
    B = np.eye(4)[None].copy()
    B[0, 2, 2] = 0.0
    g = R.features(B, 1)[0]
    assert g[1] == 1 and g[2] == 30 and g[11] == 1 and g[22] == 0.25
    # symmetric input: lower and upper Frobenius norms agree
    rng = np.random.default_rng(2)
    S = rng.normal(size=(3, 6, 6))
    S = S + S.transpose(0, 2, 1)
    assert np.allclose(R.features(S, 0)[:, 20], 0)


def test_adam_first_step_moves_by_lr():
    P = np.zeros(4)
    g = np.array([1.0, -2.0, 0.5, 0.0])
    P1, m, v = R.adam(P, g, np.zeros(4), np.zeros(4), 1, 0.1)
    assert np.allclose(P1[:3], -0.1 * np.sign(g[:3]), atol=1e-6) and P1[3] == 0


def test_selector_abi_validation_without_device():
    lib = capi.lib()
    assert lib.tsdx_cuda_selector_features_f64(None, 65, 1, None, 0, None, None) == capi.TSDX_ERR_N
    assert lib.tsdx_cuda_selector_features_f64(None, 8, -1, None, 0, None, None) == capi.TSDX_ERR_BATCH
    assert lib.tsdx_cuda_selector_features_f64(None, 8, 0, None, 0, None, None) == capi.TSDX_OK
    assert lib.tsdx_cuda_selector_features_f64(None, 8, 3, None, 0, None, None) == capi.TSDX_ERR_NULL
    assert lib.tsdx_cuda_mlp_scratch_bytes(64) == (6020 + 1) * 4
    assert lib.tsdx_cuda_mlp_scratch_bytes(65) == 2 * (6020 + 1) * 4
    assert lib.tsdx_cuda_mlp_grad(*([None] * 5), 0, None, None, None, 0, None) == capi.TSDX_ERR_BATCH
    assert lib.tsdx_cuda_mlp_forward(None, None, None, 4, None, None, None) == capi.TSDX_ERR_NULL
    assert lib.tsdx_cuda_adam_step(None, None, None, None, 4, 0.1, 0.9, 0.999, 1e-8, 0, None) == capi.TSDX_ERR_BATCH
