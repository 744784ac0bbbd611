"""B200-native batched small-matrix Cholesky / LU — a drop-in for TinySolverDx.

The NumPy-facing functions mirror TinySolverDx ``python/tinysolverdx/__init__.py``
(same names, arguments, dtype rules, return values and exceptions): inputs are
(batch, n, n) arrays (a single (n, n) matrix is also accepted) with n in 1..64;
float32 -> fp32, float64 -> fp64, float16 -> emulated fp16. ``backend="cuda"``
runs on the B200 for every function, the solves included; the CPU backends
("auto", "naive", "scalar", "simd") reproduce the reference's results bit for bit.

Beyond the reference:
  * ``gesv_ir`` / ``posv_ir``: mixed-precision factorization (fp16/bf16 tensor
    cores or fp32) with fp64 iterative refinement and an fp64 fallback;
  * ``solve_stream``: one call over an uneven stream of matrices (n 2..64, Cholesky
    and LU mixed, 1..8 right-hand sides);
  * ``selector``: the learned per-matrix precision-tier selector;
  * ``device``: the same solvers on torch CUDA tensors, stream-ordered, no copies.
"""
import numpy as np

from . import _core
from ._core import has_cuda, has_openmp, num_threads, set_num_threads, unit_roundoff  # noqa: F401
from ._core import (chol_backward_error, lu_backward_error, solve_backward_error,  # noqa: F401
                    solve_forward_error, reference_solve)

__all__ = ["cholesky", "lu", "cholesky_solve", "lu_solve", "posv", "gesv", "round_to",
           "has_cuda", "has_openmp", "num_threads", "set_num_threads", "unit_roundoff",
           "chol_backward_error", "lu_backward_error", "solve_backward_error",
           "solve_forward_error", "reference_solve", "gesv_ir", "posv_ir", "solve_stream"]

# The reference's Python layer (python/tinysolverdx/__init__.py:22-111), restated:
#   storage dtype -> implied precision: float32 fp32, float64 fp64, float16 fp16,
#     anything else TypeError (when no precision is given);
#   precision must be fp16, bf16, fp32 or fp64 (ValueError otherwise);
#   working dtype: float64 storage stays float64 whatever the precision (the core
#     rounds into the target format), any other storage is handled as float32;
#   float16 storage at precision fp16 comes back as float16;
#   a single (n, n) matrix (and its (n,) or (n, k) right-hand side) is a batch of one.
_IMPLIED_PRECISION = {np.dtype(np.float32): "fp32", np.dtype(np.float64): "fp64", np.dtype(np.float16): "fp16"}
_PRECISIONS = ("fp16", "bf16", "fp32", "fp64")
_NATIVE = {np.dtype(np.float32): "fp32", np.dtype(np.float64): "fp64"}


class _Operand:
    """A matrix argument normalised by the rules above."""

    __slots__ = ("work", "precision", "single", "storage")

    def __init__(self, a, precision):
        a = np.asarray(a)
        if precision is None:
            precision = _IMPLIED_PRECISION.get(a.dtype)
            if precision is None:
                raise TypeError(f"unsupported dtype {a.dtype}; use float16/32/64")
        elif precision not in _PRECISIONS:
            raise ValueError("precision must be one of fp16, bf16, fp32, fp64")
        self.precision = precision
        self.storage = a.dtype
        self.single = a.ndim == 2
        wide = a.dtype == np.float64
        self.work = np.ascontiguousarray(a[None] if self.single else a, dtype=np.float64 if wide else np.float32)

    def entry(self, op):
        """The core entry point of ``op`` for the working dtype."""
        return getattr(_core, op + ("_f64" if self.work.dtype == np.float64 else "_f32"))

    def native(self):
        """True when the precision is the working dtype's own (no emulation)."""
        return _NATIVE.get(self.work.dtype) == self.precision

    def cast(self, x):
        return x.astype(np.float16) if (self.precision == "fp16" and self.storage == np.float16) else x

    def unbatch(self, *results):
        return tuple(r[0] for r in results) if self.single else results

    def rhs(self, B):
        """Right-hand sides stacked as (batch, n, k) in the working dtype, and whether
        the caller passed one vector per matrix."""
        B = np.asarray(B)
        vector = B.ndim == (1 if self.single else 2)
        if vector:
            B = B[..., None]
        if self.single:
            B = B[None]
        return np.ascontiguousarray(B, dtype=self.work.dtype), vector

    def solution(self, X, vector):
        X = X[..., 0] if vector else X
        return X[0] if self.single else X


def cholesky(A, precision=None, backend="auto"):
    """Lower Cholesky factors and LAPACK-style info (0 = ok, k>0: pivot k not positive)."""
    op = _Operand(A, precision)
    L, info = op.entry("cholesky")(op.work, op.precision, backend)
    return op.unbatch(op.cast(L), info)


def lu(A, precision=None, backend="auto"):
    """Packed LU with partial pivoting: (LU, piv, info). piv is scipy/LAPACK style (0-based)."""
    op = _Operand(A, precision)
    LU, piv, info = op.entry("lu")(op.work, op.precision, backend)
    return op.unbatch(op.cast(LU), piv, info)


def cholesky_solve(L, B, precision=None, backend="auto"):
    """Solve L L^T x = B given factors from :func:`cholesky`."""
    op = _Operand(L, precision)
    rhs, vector = op.rhs(B)
    X = op.entry("cholesky_solve")(op.work, rhs, op.precision, backend)
    return op.solution(op.cast(X), vector)


def lu_solve(LU, piv, B, precision=None, backend="auto"):
    """Solve A x = B given (LU, piv) from :func:`lu`."""
    op = _Operand(LU, precision)
    p = np.asarray(piv)
    p = np.ascontiguousarray(p[None] if op.single else p, dtype=np.int32)
    rhs, vector = op.rhs(B)
    X = op.entry("lu_solve")(op.work, p, rhs, op.precision, backend)
    return op.solution(op.cast(X), vector)


def _fused(kind, A, B, precision):
    """posv/gesv on the GPU in one pass (A untouched), when the precision is native."""
    op = _Operand(A, precision)
    if not op.native():
        return None
    rhs, vector = op.rhs(B)
    X, info = op.entry(kind + "_cuda")(op.work, rhs)
    return op.solution(X, vector), (info[0] if op.single else info)


def posv(A, B, precision=None, backend="auto"):
    """Solve SPD systems A x = B. Returns (x, info)."""
    if backend == "cuda":
        r = _fused("posv", A, B, precision)
        if r is not None:
            return r
    L, info = cholesky(A, precision, backend)
    return cholesky_solve(L, B, precision, backend), info


def gesv(A, B, precision=None, backend="auto"):
    """Solve general systems A x = B with partial pivoting. Returns (x, info)."""
    if backend == "cuda":
        r = _fused("gesv", A, B, precision)
        if r is not None:
            return r
    LU, piv, info = lu(A, precision, backend)
    return lu_solve(LU, piv, B, precision, backend), info


def round_to(x, precision):
    """Round values to the nearest number representable in ``precision`` (float64 in/out)."""
    return _core.round_to_f64(np.ascontiguousarray(x, dtype=np.float64), precision)


# ---- mixed precision + iterative refinement ------------------------------------------
TIERS = {"fp16": 0, "bf16": 1, "fp32": 2, "fp64": 3}


def _ir(spd, A, b, tier, itmax, tol):
    import torch
    from . import device
    A = np.ascontiguousarray(A, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    single = A.ndim == 2
    if single:
        A, b = A[None], b[None]
    if A.ndim != 3 or A.shape[1] != A.shape[2] or b.shape != A.shape[:2]:
        raise ValueError("expected A (batch, n, n) and b (batch, n)")
    a = torch.from_numpy(A).cuda()
    x = torch.from_numpy(b).cuda()
    t = None
    default = 2
    if isinstance(tier, str):
        default = TIERS[tier]
    elif tier is not None:
        t = torch.as_tensor(np.asarray(tier, dtype=np.int8)).cuda()
    info, status, bwd = device.ir(a, x, spd, tier=t, default_tier=default, itmax=itmax, tol=tol)
    out = (x.cpu().numpy(), info.cpu().numpy(), status.cpu().numpy(), bwd.cpu().numpy())
    return tuple(o[0] for o in out) if single else out


def gesv_ir(A, b, tier="fp32", itmax=3, tol=1e-15):
    """Mixed-precision LU + fp64 iterative refinement (float64 A, one right-hand side).

    ``tier`` is "fp16", "bf16", "fp32", "fp64" or a per-matrix int8 array (0..3).
    Returns (x, info, status, bwd): status >= 0 is the number of refinement steps,
    -1 means the matrix was re-solved by the plain fp64 path."""
    return _ir(False, A, b, tier, itmax, tol)


def posv_ir(A, b, tier="fp32", itmax=3, tol=1e-15):
    """Mixed-precision Cholesky + fp64 iterative refinement (SPD float64 A)."""
    return _ir(True, A, b, tier, itmax, tol)


def solve_stream(mats, rhs, kinds, write_factors=False):
    """Solve a ragged list of systems with the uneven-stream kernels in one call.

    mats: sequence of (n_i, n_i) float32 or float64 arrays (one dtype for all), n_i in 1..64;
    rhs: sequence of (n_i,) or (n_i, k_i) arrays, k_i in 0..8 (None -> no right-hand side);
    kinds: sequence of "cholesky"/"lu" (or 0/1). Returns (X list, info array), plus
    (factors list, pivots list) when write_factors. Factors, pivots, info and X are
    bit-identical to ``posv``/``gesv`` with backend="cuda" on each matrix. The set moves
    through the device in chunks of about 96 MB, so it may exceed device memory.
    NumPy arrays are pageable host memory: a copy between them and the device returns
    only when it is done, so from here the chunks run one after another, without the
    copy/compute overlap that ``stream.solve_host`` reaches on pinned torch tensors.
    """
    import torch
    from . import stream as _stream
    if not has_cuda():
        raise RuntimeError("solve_stream needs the CUDA backend")
    count = len(mats)
    if not (len(rhs) == count == len(kinds)):
        raise ValueError("mats, rhs and kinds must have the same length")
    if count == 0:
        return ([], np.zeros(0, np.int32)) + (([], []) if write_factors else ())
    dt = np.asarray(mats[0]).dtype
    if dt not in (np.float32, np.float64):
        raise TypeError("solve_stream takes float32 or float64 matrices")
    kind = np.array([k if isinstance(k, (int, np.integer)) else {"cholesky": 0, "lu": 1}[k] for k in kinds], np.int8)
    ns = np.array([np.asarray(a).shape[0] for a in mats], np.int32)
    vec, bs = [], []
    for a, b, n in zip(mats, rhs, ns):
        a = np.asarray(a)
        if a.shape != (n, n) or a.dtype != dt:
            raise ValueError("every matrix must be square and of the first matrix's dtype")
        if not 1 <= n <= 64:
            raise ValueError("matrix size n outside supported range [1, 64]")
        b = np.zeros((n, 0), dt) if b is None else np.asarray(b, dt)
        vec.append(b.ndim == 1)
        b = b.reshape(n, -1)
        if b.shape[1] > 8:
            raise ValueError("at most 8 right-hand sides per matrix")
        bs.append(b)
    nrhs = np.array([b.shape[1] for b in bs], np.int32)
    aoff, boff, poff, *_ = _stream.layout(ns, nrhs)
    # the host-memory stream call moves the set through the device in chunks, so the set
    # may be larger than device memory
    A = torch.from_numpy(np.concatenate([np.ascontiguousarray(a).ravel() for a in mats]))
    Bh = np.concatenate([b.ravel() for b in bs])
    B = torch.from_numpy(Bh if Bh.size else np.zeros(1, dt))
    piv = torch.zeros(int(ns.sum()), dtype=torch.int32)
    info = torch.zeros(count, dtype=torch.int32)
    _stream.solve_host(A, B, piv, info, torch.from_numpy(np.ascontiguousarray(ns, np.int32)),
                       torch.from_numpy(np.ascontiguousarray(nrhs, np.int32)),
                       torch.from_numpy(np.ascontiguousarray(kind, np.int8)), write_factors=write_factors)
    Xh, infoh = B.numpy(), info.numpy()
    X = []
    for i, (n, k) in enumerate(zip(ns, nrhs)):
        x = Xh[boff[i]:boff[i] + n * k].reshape(n, k)
        X.append(x[:, 0].copy() if vec[i] else x.copy())
    if not write_factors:
        return X, infoh
    Ah, ph = A.numpy(), piv.numpy()
    F = [Ah[aoff[i]:aoff[i] + n * n].reshape(n, n).copy() for i, n in enumerate(ns)]
    P = [ph[poff[i]:poff[i] + n].copy() if kind[i] else None for i, n in enumerate(ns)]
    return X, infoh, F, P
