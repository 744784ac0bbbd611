"""The solvers on torch CUDA tensors: in place, stream-ordered, no host copies.

Thin wrappers over the device-pointer C-ABI (include/tsdx_cuda.h). Inputs must be
contiguous float32/float64 CUDA tensors; pivots and info are int32 tensors.
"""
import torch

from . import capi


def _check(t, name, dtype=None):
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}")


def _i32(shape, like):
    return torch.zeros(shape, dtype=torch.int32, device=like.device)


def potrf(A, stream=None):
    """A <- L (lower, upper zeroed). Returns info."""
    _check(A, "A")
    info = _i32(A.shape[0], A)
    capi.potrf(A, info, stream)
    return info


def getrf(A, stream=None):
    """A <- L\\U. Returns (piv, info)."""
    _check(A, "A")
    piv, info = _i32(A.shape[:2], A), _i32(A.shape[0], A)
    capi.getrf(A, piv, info, stream)
    return piv, info


def potrs(L, B, stream=None):
    """B <- (L L^T)^{-1} B."""
    _check(L, "L")
    _check(B, "B", L.dtype)
    capi.potrs(L, B, stream)


def getrs(LU, piv, B, stream=None):
    """B <- (P L U)^{-1} B."""
    _check(LU, "LU")
    _check(B, "B", LU.dtype)
    capi.getrs(LU, piv, B, stream)


def posv(A, B, stream=None):
    """A <- L, B <- X. Returns info."""
    _check(A, "A")
    _check(B, "B", A.dtype)
    info = _i32(A.shape[0], A)
    capi.posv(A, B, info, stream)
    return info


def gesv(A, B, stream=None):
    """A <- L\\U, B <- X. Returns (piv, info)."""
    _check(A, "A")
    _check(B, "B", A.dtype)
    piv, info = _i32(A.shape[:2], A), _i32(A.shape[0], A)
    capi.gesv(A, B, piv, info, stream)
    return piv, info


def ir(A, x, spd, tier=None, default_tier=2, itmax=3, tol=1e-15, stream=None):
    """Mixed-precision solve with fp64 refinement: x (batch, n) holds b on entry and
    the solution on exit; A (float64) is not modified. tier: optional int8 tensor.
    Returns (info, status, bwd)."""
    _check(A, "A", torch.float64)
    _check(x, "x", torch.float64)
    batch, n = A.shape[0], A.shape[-1]
    info, status = _i32(batch, A), _i32(batch, A)
    bwd = torch.zeros(batch, dtype=torch.float64, device=A.device)
    name = "tsdx_cuda_posv_ir_f64" if spd else "tsdx_cuda_gesv_ir_f64"
    capi.check(capi.call(name, capi.ptr(A), n, batch, capi.ptr(x), capi.ptr(tier), int(default_tier), int(itmax),
                         float(tol), capi.ptr(info), capi.ptr(status), capi.ptr(bwd), capi.stream_ptr(stream)), name)
    return info, status, bwd


def _metric_out(A):
    return torch.empty(A.shape[0], dtype=torch.float64, device=A.device)


def solve_backward_error(A, x, b, stream=None):
    """||b - A x|| / (||A||_F ||x|| + ||b||) per matrix, double-double on the device
    (the reference's runtime.cpp:230-242 metric). A (batch, n, n), x and b (batch, n), float64."""
    for t, nm in ((A, "A"), (x, "x"), (b, "b")):
        _check(t, nm, torch.float64)
    out = _metric_out(A)
    capi.check(capi.call("tsdx_cuda_solve_backward_error_f64", capi.ptr(A), capi.ptr(x), capi.ptr(b), A.shape[-1],
                         A.shape[0], capi.ptr(out), capi.stream_ptr(stream)), "solve_backward_error")
    return out


def lu_backward_error(A, LU, piv, stream=None):
    """||P A - L U||_F / ||A||_F per matrix (runtime.cpp:208-228), double-double on the device."""
    _check(A, "A", torch.float64)
    _check(LU, "LU", torch.float64)
    _check(piv, "piv", torch.int32)
    out = _metric_out(A)
    capi.check(capi.call("tsdx_cuda_lu_backward_error_f64", capi.ptr(A), capi.ptr(LU), capi.ptr(piv), A.shape[-1],
                         A.shape[0], capi.ptr(out), capi.stream_ptr(stream)), "lu_backward_error")
    return out


def chol_backward_error(A, L, stream=None):
    """||A - L L^T||_F / ||A||_F per matrix (runtime.cpp:194-206), double-double on the device."""
    _check(A, "A", torch.float64)
    _check(L, "L", torch.float64)
    out = _metric_out(A)
    capi.check(capi.call("tsdx_cuda_chol_backward_error_f64", capi.ptr(A), capi.ptr(L), A.shape[-1], A.shape[0],
                         capi.ptr(out), capi.stream_ptr(stream)), "chol_backward_error")
    return out
