"""tsdx_cuda_solve_stream_noalloc_f32 (scratch in a fixed device array, no
allocation) against tsdx_cuda_solve_stream_f32 with caller scratch: two calls in a
row on one CUDA stream, each over a different set of matrices, bit-identical
factors, pivots, info and X; the calls leave the device's memory pool untouched;
a count above the fixed capacity is rejected before anything runs.

The entry point exists for callers that may not allocate device memory when they
call (their memory belongs to another allocator, or an allocation could stall or
fail mid-request); the second call checks that nothing left in the shared array by
the first call leaks into its results.

Kept in its own file, named to be collected last, so that it also runs after every
other test has used the library on the same device."""
import ctypes

import numpy as np
import pytest

from conftest import load_pkg

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

capi = load_pkg("capi")
stream = load_pkg("stream")
matrices = load_pkg("matrices")

CAPACITY = 1 << 18


def packed(seed, count):
    r = np.random.default_rng(seed)
    n = r.integers(1, 65, count).astype(np.int32)
    kind = r.integers(0, 2, count).astype(np.int8)
    nrhs = r.choice([0, 1, 2, 4, 8], count).astype(np.int32)
    aoff, boff, poff, na, nb, npv = stream.layout(n, nrhs)
    A = torch.empty(na, dtype=torch.float32)
    for i in range(count):
        gen = matrices.spd if kind[i] == 0 else matrices.general
        A[aoff[i]:aoff[i] + n[i] * n[i]] = torch.from_numpy(gen(r, 1, int(n[i]), 1e4)[0].astype(np.float32).ravel())
    B = torch.from_numpy(r.standard_normal(max(nb, 1)).astype(np.float32))
    d = "cuda"
    meta = [torch.from_numpy(x).to(d) for x in (n, nrhs, kind)] + [t.to(d) for t in (aoff, boff, poff)]
    return A.to(d), B.to(d), max(npv, 1), meta


def run(entry, A, B, npv, meta, wf):
    n, nrhs, kind, aoff, boff, poff = meta
    A, B = A.clone(), B.clone()
    piv = torch.zeros(npv, dtype=torch.int32, device="cuda")
    info = torch.full((n.numel(),), 99, dtype=torch.int32, device="cuda")
    P = capi.ptr
    if entry == "noalloc":
        rc = capi.call("tsdx_cuda_solve_stream_noalloc_f32", P(A), P(aoff), P(B), P(boff), P(piv), P(poff), P(info),
                       P(n), P(nrhs), P(kind), n.numel(), wf, 0, capi.stream_ptr())
    else:
        sc = torch.empty(stream.scratch_bytes(n.numel()), dtype=torch.uint8, device="cuda")
        rc = capi.call("tsdx_cuda_solve_stream_f32", P(A), P(aoff), P(B), P(boff), P(piv), P(poff), P(info), P(n),
                       P(nrhs), P(kind), n.numel(), wf, 0, P(sc), sc.numel(), capi.stream_ptr())
    capi.check(rc, entry)
    torch.cuda.synchronize()
    return A, B, piv, info


class PoolWatch:
    """High-water mark of the device's default memory pool (cudaMallocAsync's pool),
    reset before the watched calls: any stream-ordered allocation shows up in it."""

    USED_MEM_HIGH = 0x8  # cudaMemPoolAttrUsedMemHigh

    def __init__(self):
        self.rt = ctypes.CDLL("libcudart.so.12")
        self.pool = ctypes.c_void_p()
        assert self.rt.cudaDeviceGetDefaultMemPool(ctypes.byref(self.pool), torch.cuda.current_device()) == 0

    def reset(self):
        zero = ctypes.c_uint64(0)
        assert self.rt.cudaMemPoolSetAttribute(self.pool, self.USED_MEM_HIGH, ctypes.byref(zero)) == 0

    def high(self):
        v = ctypes.c_uint64(0)
        assert self.rt.cudaMemPoolGetAttribute(self.pool, self.USED_MEM_HIGH, ctypes.byref(v)) == 0
        return v.value


def test_noalloc_matches_scratch_entry_two_calls_in_a_row():
    for seed, count, wf in ((1, 3000, 1), (2, 1700, 0)):
        A, B, npv, meta = packed(seed, count)
        ref = run("scratch", A, B, npv, meta, wf)
        watch = PoolWatch()
        torch.cuda.synchronize()
        watch.reset()
        got = run("noalloc", A, B, npv, meta, wf)
        assert watch.high() == 0, "the no-allocation entry point allocated from the device pool"
        assert (got[3] != 99).all()
        for x, y in zip(ref, got):
            assert torch.equal(x.view(torch.int32) if x.dtype == torch.float32 else x,
                               y.view(torch.int32) if y.dtype == torch.float32 else y)


def test_pool_watch_sees_a_stream_allocation():
    """The pool check above can fail: the same solve without caller scratch takes its
    scratch from the device pool, and the high-water mark shows it."""
    A, B, npv, meta = packed(3, 500)
    n, nrhs, kind, aoff, boff, poff = meta
    piv = torch.zeros(npv, dtype=torch.int32, device="cuda")
    info = torch.zeros(n.numel(), dtype=torch.int32, device="cuda")
    watch = PoolWatch()
    torch.cuda.synchronize()
    watch.reset()
    P = capi.ptr
    rc = capi.call("tsdx_cuda_solve_stream_f32", P(A), P(aoff), P(B), P(boff), P(piv), P(poff), P(info), P(n),
                   P(nrhs), P(kind), n.numel(), 1, 0, None, 0, capi.stream_ptr())
    capi.check(rc, "stream without scratch")
    torch.cuda.synchronize()
    assert watch.high() > 0


def test_noalloc_rejects_count_above_capacity():
    count = CAPACITY + 1
    d = "cuda"
    n = torch.ones(count, dtype=torch.int32, device=d)
    nrhs = torch.ones(count, dtype=torch.int32, device=d)
    kind = torch.ones(count, dtype=torch.int8, device=d)
    off = torch.arange(count, dtype=torch.int64, device=d)
    A = torch.full((count,), 2.0, device=d)
    B = torch.ones(count, device=d)
    piv = torch.zeros(count, dtype=torch.int32, device=d)
    info = torch.full((count,), 99, dtype=torch.int32, device=d)
    P = capi.ptr
    rc = capi.call("tsdx_cuda_solve_stream_noalloc_f32", P(A), P(off), P(B), P(off), P(piv), P(off), P(info), P(n),
                   P(nrhs), P(kind), count, 1, 0, capi.stream_ptr())
    torch.cuda.synchronize()
    assert rc == capi.TSDX_ERR_TOO_LARGE
    assert "262144" in capi.last_error()
    assert (info == 99).all() and (B == 1).all()  # nothing ran
    # at the capacity itself the call runs (n = 1: x = 1/2)
    rc = capi.call("tsdx_cuda_solve_stream_noalloc_f32", P(A), P(off), P(B), P(off), P(piv), P(off), P(info), P(n),
                   P(nrhs), P(kind), CAPACITY, 1, 0, capi.stream_ptr())
    torch.cuda.synchronize()
    assert rc == 0
    assert (info[:CAPACITY] == 0).all() and (B[:CAPACITY] == 0.5).all() and (B[CAPACITY:] == 1).all()
