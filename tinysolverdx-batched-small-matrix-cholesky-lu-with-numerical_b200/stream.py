"""Uneven batched stream: one call over a ragged list of matrices on torch CUDA tensors.

Matrices of mixed order n (1..64), Cholesky (posv) and LU (gesv) mixed and 0..8
right-hand sides each are packed back to back in flat buffers and solved by one
counting sort into size buckets plus persistent kernels that drain them, one per order class
(tsdx_cuda_solve_stream_* in include/tsdx_cuda.h). The results are bit-identical
to the dense posv/gesv of each matrix.

TinySolverDx itself has no such call (its batched entry points take one
(batch, n, n) stack of equal n, cpp/include/tinysolverdx/batched.hpp:112-181); this
module is the mixed-workload path on top of the same per-matrix solvers.

``StreamPlan`` fixes a layout once, picks the fastest warp schedule for it by timing
the candidates on the device (the autotuner), captures the launches of a solve
in a CUDA graph and replays it on new data.
"""
import torch

from . import capi

CHOLESKY, LU = 0, 1
# sched bit c (order class c: n in 1..8, 9..16, 17..24, 25..32) set -> those matrices
# run one per warp; clear -> they share a warp (8 Cholesky or 4 LU at n <= 8, 4 at
# n <= 16, 4 (float32) or 2 (float64) at n <= 24, 2 at n <= 32)
SCHED_BITS = 4


def layout(n, nrhs, device=None):
    """Packed element offsets for matrices of order n[i] with nrhs[i] right-hand sides.

    Returns (aoff, boff, poff, a_elems, b_elems, p_elems); offsets are int64 tensors.
    """
    n = torch.as_tensor(n, dtype=torch.int64, device=device)
    nrhs = torch.as_tensor(nrhs, dtype=torch.int64, device=device)

    def excl(x):
        c = torch.cumsum(x, 0)
        return c - x, int(c[-1]) if len(c) else 0

    aoff, na = excl(n * n)
    boff, nb = excl(n * nrhs)
    poff, npv = excl(n)
    return aoff, boff, poff, na, nb, npv


def scratch_bytes(count):
    return int(capi.call("tsdx_cuda_stream_scratch_bytes", int(count)))


def _check(t, name, dtype=None):
    if t is None:
        return
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, not {t.dtype}")


def solve(A, aoff, B, boff, piv, poff, info, n, nrhs, kind, write_factors=True, sched=0, scratch=None,
          stream=None):
    """Solve every matrix of a packed stream in place (stream-ordered, no host sync).

    A: flat float32/float64 (matrix i at aoff[i], n[i] x n[i] row-major) -> factors
    B: flat, same dtype (matrix i's n[i] x nrhs[i] right-hand sides at boff[i]) -> X; may be None
    piv: flat int32 (n[i] LU pivots at poff[i]); required when write_factors
    info: int32 (count,) -> LAPACK info, -1 for an entry outside n in [1, 64], nrhs in [0, 8]
    n, nrhs: int32 (count,); kind: int8 (count,) 0 = Cholesky, nonzero = LU
    scratch: uint8 CUDA tensor of at least scratch_bytes(count) bytes, or None
    (then it is allocated on the stream for this call).
    """
    _check(A, "A")
    if A.dtype not in (torch.float32, torch.float64):
        raise TypeError("A must be float32 or float64")
    _check(B, "B", A.dtype)
    for t, nm in ((aoff, "aoff"), (boff, "boff"), (poff, "poff")):
        _check(t, nm, torch.int64)
    for t, nm in ((piv, "piv"), (info, "info"), (n, "n"), (nrhs, "nrhs")):
        _check(t, nm, torch.int32)
    _check(kind, "kind", torch.int8)
    count = n.numel()
    if scratch is not None:
        _check(scratch, "scratch")
    name = f"tsdx_cuda_solve_stream_{capi.sfx(A.dtype)}"
    P = capi.ptr
    capi.check(capi.call(name, P(A), P(aoff), P(B), P(boff), P(piv), P(poff), P(info), P(n), P(nrhs), P(kind),
                         count, int(bool(write_factors)), int(sched), P(scratch),
                         scratch.numel() * scratch.element_size() if scratch is not None else 0,
                         capi.stream_ptr(stream)), name)


def _check_host(t, name, dtype=None):
    if t is None:
        return
    if t.is_cuda or not t.is_contiguous():
        raise ValueError(f"{name} must be a contiguous CPU tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, not {t.dtype}")


def solve_host(A, B, piv, info, n, nrhs, kind, write_factors=True, sched=0):
    """Solve a packed stream held in host memory, in place (synchronous).

    Same arguments as ``solve`` without the offsets, all CPU tensors: the matrices
    are packed back to back in index order (``layout``'s offsets). The library moves
    the set through the device in chunks of about 96 MB with the copies of one
    chunk overlapping the solve of the next, so the device never holds the whole set.
    Pin A, B, piv and info (``tensor.pin_memory()``) for the copies to overlap.
    Raises on n outside [1, 64] or nrhs outside [0, 8] before anything is copied.
    """
    _check_host(A, "A")
    if A.dtype not in (torch.float32, torch.float64):
        raise TypeError("A must be float32 or float64")
    _check_host(B, "B", A.dtype)
    for t, nm in ((piv, "piv"), (info, "info"), (n, "n"), (nrhs, "nrhs")):
        _check_host(t, nm, torch.int32)
    _check_host(kind, "kind", torch.int8)
    count = n.numel()
    if nrhs.numel() != count or kind.numel() != count or (info is not None and info.numel() < count):
        raise ValueError("n, nrhs, kind and info must have one entry per matrix")
    _, _, _, na, nb, npv = layout(n, nrhs)
    if A.numel() < na or (nb and (B is None or B.numel() < nb)) or (write_factors and (piv is None or piv.numel() < npv)):
        raise ValueError("A, B or piv smaller than the packed layout of n and nrhs")
    name = f"tsdx_cuda_solve_stream_host_{capi.sfx(A.dtype)}"
    P = capi.ptr
    capi.check(capi.call(name, P(A), P(B), P(piv), P(info), P(n), P(nrhs), P(kind), count,
                         int(bool(write_factors)), int(sched)), name)


class StreamPlan:
    """A fixed stream layout with device buffers, a tuned schedule and a CUDA graph.

    n, nrhs, kind: per-matrix order, right-hand-side count and kind (CHOLESKY / LU).
    Fill ``plan.A`` / ``plan.B`` (see ``load``), call ``run()``; results are in
    ``plan.A`` (factors, when write_factors), ``plan.B`` (X), ``plan.piv``, ``plan.info``.
    """

    def __init__(self, n, nrhs, kind, dtype=torch.float32, device="cuda", write_factors=True):
        self.device = torch.device(device)
        self.count = len(n)
        self.n = torch.as_tensor(n, dtype=torch.int32).to(self.device)
        self.nrhs = torch.as_tensor(nrhs, dtype=torch.int32).to(self.device)
        self.kind = torch.as_tensor(kind, dtype=torch.int8).to(self.device)
        self.aoff, self.boff, self.poff, na, nb, npv = layout(self.n.cpu(), self.nrhs.cpu())
        self.aoff, self.boff, self.poff = (t.to(self.device) for t in (self.aoff, self.boff, self.poff))
        self.A = torch.zeros(max(na, 1), dtype=dtype, device=self.device)
        self.B = torch.zeros(max(nb, 1), dtype=dtype, device=self.device)
        self.piv = torch.zeros(max(npv, 1), dtype=torch.int32, device=self.device)
        self.info = torch.zeros(max(self.count, 1), dtype=torch.int32, device=self.device)
        self.scratch = torch.empty(scratch_bytes(self.count), dtype=torch.uint8, device=self.device)
        self.write_factors = write_factors
        self.sched = 0
        self.timings = {}
        self.graph = None

    def load(self, A, B):
        """Copy packed inputs (flat tensors, any device) into the plan's buffers."""
        if A.numel() > self.A.numel() or B.numel() > self.B.numel():
            raise ValueError("inputs larger than the plan's layout")
        self.A[:A.numel()].copy_(A.reshape(-1), non_blocking=True)
        self.B[:B.numel()].copy_(B.reshape(-1), non_blocking=True)

    def launch(self, sched=None, stream=None):
        solve(self.A, self.aoff, self.B, self.boff, self.piv, self.poff, self.info, self.n, self.nrhs, self.kind,
              self.write_factors, self.sched if sched is None else sched, self.scratch, stream)

    def _time(self, A0, B0, sched, reps):
        s = torch.cuda.current_stream(self.device)
        best = float("inf")
        for _ in range(reps):
            self.load(A0, B0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(s)
            self.launch(sched, s)
            e1.record(s)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        self.timings[sched] = best
        return best

    def tune(self, A, B, reps=3):
        """Pick the warp schedule: starting from all-packed, flip each order class to
        one matrix per warp in turn and keep the flip when it times faster on (A, B)."""
        A0, B0 = A.reshape(-1).to(self.device), B.reshape(-1).to(self.device)
        self.timings = {}
        sched = 0
        best = self._time(A0, B0, sched, reps)
        for c in range(SCHED_BITS):
            t = self._time(A0, B0, sched | (1 << c), reps)
            if t < best:
                sched, best = sched | (1 << c), t
        self.sched = sched
        self.graph = None
        return self.sched

    def capture(self):
        """Capture one solve (memset, histogram, scan, scatter, memset, seven drains) in a CUDA graph."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.launch(stream=s)  # warm-up outside the capture (function attributes, occupancy)
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.launch(stream=torch.cuda.current_stream(self.device))
        self.graph = g
        return g

    def run(self):
        if self.graph is None:
            self.capture()
        self.graph.replay()
