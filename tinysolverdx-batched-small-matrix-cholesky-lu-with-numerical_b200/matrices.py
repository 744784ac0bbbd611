"""Seeded test-matrix generators with a prescribed 2-norm condition number.

Same construction as TinySolverDx ``python/tinysolverdx/matrices.py:5-21``
(Q from the QR of an N(0,1) matrix with the sign of diag(R) folded in;
SPD = Q diag(lambda) Q^T symmetrised, general = U diag(sigma) V^T, spectra
geometric from 1 down to 1/kappa), extended so that ``kappa`` may be one value
per matrix, plus the workload builders for the benchmark configurations.
Called with a scalar ``kappa`` and the same ``rng`` the functions return exactly
the reference generator's matrices.
"""
import numpy as np


def _orthogonal(rng, batch, n):
    q, r = np.linalg.qr(rng.standard_normal((batch, n, n)))
    return q * np.sign(np.diagonal(r, axis1=1, axis2=2))[:, None, :]


def _spectrum(batch, n, kappa):
    k = np.asarray(kappa, dtype=np.float64)
    if k.ndim == 0:
        return np.broadcast_to(np.geomspace(1.0, 1.0 / float(k), n), (batch, n))
    # per-matrix geometric spectrum 1 .. 1/kappa_b
    t = np.linspace(0.0, 1.0, n) if n > 1 else np.zeros(1)
    return np.exp(-np.log(k)[:, None] * t[None, :])


def spd(rng, batch, n, kappa):
    """SPD matrices Q diag(lambda) Q^T with eigenvalues geometric in [1/kappa, 1]."""
    lam = _spectrum(batch, n, kappa)
    Q = _orthogonal(rng, batch, n)
    A = np.einsum("bij,bj,bkj->bik", Q, lam, Q)
    return (A + A.transpose(0, 2, 1)) / 2


def general(rng, batch, n, kappa):
    """General matrices U diag(sigma) V^T with singular values geometric in [1/kappa, 1]."""
    s = _spectrum(batch, n, kappa)
    return np.einsum("bij,bj,bkj->bik", _orthogonal(rng, batch, n), s, _orthogonal(rng, batch, n))


def log_uniform(rng, size, lo, hi):
    """kappa drawn log-uniformly in [lo, hi]."""
    return np.exp(rng.uniform(np.log(lo), np.log(hi), size))


def zero_one_column(rng, A, frac):
    """Zero one random column in a random ``frac`` of the matrices (singular -> info > 0)."""
    batch, n = A.shape[0], A.shape[1]
    pick = rng.random(batch) < frac
    cols = rng.integers(0, n, batch)
    idx = np.nonzero(pick)[0]
    A[idx, :, cols[idx]] = 0.0
    return pick


# ---- torch generators for the large benchmark stacks (same construction) -----
def torch_orthogonal(gen, batch, n, device, dtype):
    import torch
    x = torch.randn(batch, n, n, generator=gen, device=device, dtype=torch.float64)
    q, r = torch.linalg.qr(x)
    return (q * torch.sign(torch.diagonal(r, dim1=1, dim2=2))[:, None, :]).to(dtype)


def torch_stack(kind, n, batch, kappa_lo, kappa_hi, seed, device="cuda", dtype=None, chunk=16384):
    """(batch, n, n) float64 stack of SPD ("spd") or general ("general") matrices with
    kappa log-uniform in [kappa_lo, kappa_hi], built on ``device`` in chunks."""
    import torch
    dtype = dtype or torch.float64
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    out = torch.empty(batch, n, n, device=device, dtype=torch.float64)
    t = torch.linspace(0.0, 1.0, n, device=device, dtype=torch.float64) if n > 1 else torch.zeros(1, device=device, dtype=torch.float64)
    for s in range(0, batch, chunk):
        b = min(chunk, batch - s)
        u = torch.rand(b, generator=gen, device=device, dtype=torch.float64)
        logk = np.log(kappa_lo) + u * (np.log(kappa_hi) - np.log(kappa_lo))
        lam = torch.exp(-logk[:, None] * t[None, :])
        Q = torch_orthogonal(gen, b, n, device, torch.float64)
        if kind == "spd":
            A = torch.einsum("bij,bj,bkj->bik", Q, lam, Q)
            A = (A + A.transpose(1, 2)) / 2
        else:
            V = torch_orthogonal(gen, b, n, device, torch.float64)
            A = torch.einsum("bij,bj,bkj->bik", Q, lam, V)
        out[s:s + b] = A
    return out.to(dtype)
