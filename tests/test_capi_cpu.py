"""The C-ABI library loads without a GPU, exports every symbol include/tsdx_cuda.h
declares, and rejects bad arguments before touching a device (the reference's
batched.hpp:39-43, :184 validation)."""
import ctypes as C
import re

import numpy as np

from conftest import ROOT, load_pkg

capi = load_pkg("capi")


def declared_symbols():
    text = (ROOT / "include" / "tsdx_cuda.h").read_text()
    return sorted(set(re.findall(r"\b(tsdx_cuda_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = capi.lib()
    names = declared_symbols()
    assert len(names) >= 27
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) >= {k for k in capi.SIGNATURES if not k.startswith("tsdx_internal_")}


def test_validation_without_device():
    lib = capi.lib()
    A = np.zeros((2, 4, 4))
    info = np.zeros(2, np.int32)
    piv = np.zeros((2, 4), np.int32)
    assert lib.tsdx_cuda_cholesky_batched_host_f64(capi.ptr(A), 0, 2, capi.ptr(info)) == capi.TSDX_ERR_N
    assert lib.tsdx_cuda_cholesky_batched_host_f64(capi.ptr(A), 65, 2, capi.ptr(info)) == capi.TSDX_ERR_N
    assert lib.tsdx_cuda_cholesky_batched_host_f64(capi.ptr(A), 4, -1, capi.ptr(info)) == capi.TSDX_ERR_BATCH
    assert lib.tsdx_cuda_lu_batched_host_f64(capi.ptr(A), 4, 2, None, capi.ptr(info)) == capi.TSDX_ERR_NULL
    assert lib.tsdx_cuda_posv_batched_host_f64(capi.ptr(A), 4, 2, capi.ptr(A), -1, capi.ptr(info)) == capi.TSDX_ERR_NRHS
    # an empty batch is a successful no-op (batched.hpp:126)
    assert lib.tsdx_cuda_lu_batched_host_f64(capi.ptr(A), 4, 0, capi.ptr(piv), capi.ptr(info)) == capi.TSDX_OK
    assert lib.tsdx_cuda_getrf_f32(None, 4, 0, None, None, None) == capi.TSDX_ERR_NULL


def test_stream_validation_without_device():
    lib = capi.lib()
    assert lib.tsdx_cuda_stream_scratch_bytes(10) == (4 * 32 + 2 + 10) * 4
    assert lib.tsdx_cuda_stream_scratch_bytes(-1) == 0
    nul = [None] * 10
    assert lib.tsdx_cuda_solve_stream_f32(*nul, 0, 1, 0, None, 0, None) == capi.TSDX_OK
    assert lib.tsdx_cuda_solve_stream_f64(*nul, -1, 1, 0, None, 0, None) == capi.TSDX_ERR_BATCH
    assert lib.tsdx_cuda_solve_stream_f32(*nul, 5, 1, 0, None, 0, None) == capi.TSDX_ERR_NULL
    # the no-allocation variant rejects a count above its fixed capacity first
    assert lib.tsdx_cuda_solve_stream_noalloc_f32(*nul, (1 << 18) + 1, 1, 0, None) == capi.TSDX_ERR_TOO_LARGE
    assert "262144" in capi.last_error()
    assert lib.tsdx_cuda_solve_stream_noalloc_f32(*nul, -3, 1, 0, None) == capi.TSDX_ERR_BATCH
    assert lib.tsdx_cuda_solve_stream_noalloc_f32(*nul, 0, 1, 0, None) == capi.TSDX_OK
    # host-memory stream: every entry is checked before any CUDA call
    import numpy as np
    nn = np.array([3, 65], np.int32)
    rr = np.array([1, 1], np.int32)
    kk = np.zeros(2, np.int8)
    A = np.zeros(9 + 65 * 65, np.float32)
    B = np.zeros(3 + 65, np.float32)
    pv = np.zeros(68, np.int32)
    f = lib.tsdx_cuda_solve_stream_host_f32
    P = capi.ptr
    assert f(P(A), P(B), P(pv), None, P(nn), P(rr), P(kk), 2, 1, 0) == capi.TSDX_ERR_N
    nn[1] = 2
    rr[0] = 9
    assert f(P(A), P(B), P(pv), None, P(nn), P(rr), P(kk), 2, 1, 0) == capi.TSDX_ERR_NRHS
    rr[0] = 1
    assert f(P(A), None, P(pv), None, P(nn), P(rr), P(kk), 2, 1, 0) == capi.TSDX_ERR_NULL  # B with nrhs > 0
    assert f(P(A), P(B), None, None, P(nn), P(rr), P(kk), 2, 1, 0) == capi.TSDX_ERR_NULL  # piv with factors
    assert f(None, P(B), P(pv), None, P(nn), P(rr), P(kk), 2, 1, 0) == capi.TSDX_ERR_NULL
    assert lib.tsdx_cuda_solve_stream_host_f64(None, None, None, None, None, None, None, -1, 1, 0) == capi.TSDX_ERR_BATCH
    assert lib.tsdx_cuda_solve_stream_host_f64(None, None, None, None, None, None, None, 0, 1, 0) == capi.TSDX_OK


def test_stream_solve_host_python_validation():
    """stream.solve_host rejects device tensors, wrong dtypes and buffers smaller than
    the packed layout before calling the library; valid empty input is a no-op."""
    import pytest
    torch = pytest.importorskip("torch")
    stream = load_pkg("stream")
    n = torch.tensor([3, 2], dtype=torch.int32)
    r = torch.tensor([1, 0], dtype=torch.int32)
    k = torch.tensor([0, 1], dtype=torch.int8)
    A = torch.zeros(13, dtype=torch.float64)
    B = torch.zeros(3, dtype=torch.float64)
    piv = torch.zeros(5, dtype=torch.int32)
    info = torch.zeros(2, dtype=torch.int32)
    with pytest.raises(ValueError):  # A one element short of 3*3 + 2*2
        stream.solve_host(A[:12], B, piv, info, n, r, k)
    with pytest.raises(ValueError):  # pivots short of 3 + 2
        stream.solve_host(A, B, piv[:4], info, n, r, k)
    with pytest.raises(ValueError):  # B missing while a matrix has a right-hand side
        stream.solve_host(A, None, piv, info, n, r, k)
    with pytest.raises(TypeError):
        stream.solve_host(A, B.float(), piv, info, n, r, k)
    with pytest.raises(TypeError):
        stream.solve_host(A, B, piv, info, n.long(), r, k)
    with pytest.raises(ValueError):
        stream.solve_host(A, B, piv, info[:1], n, r, k)
    e = torch.zeros(0, dtype=torch.int32)
    stream.solve_host(A, B, piv, info, e, e, torch.zeros(0, dtype=torch.int8))  # count 0: nothing to do
