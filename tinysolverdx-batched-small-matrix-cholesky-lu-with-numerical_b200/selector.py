"""Learned per-matrix precision-tier selector for the mixed-precision solves.

A small MLP (24 features -> 64 -> 64 -> 4 tiers) predicts, per matrix, the
lowest-precision tier of {fp16, bf16, fp32, fp64} whose iterative refinement
converges (status >= 0 within ``itmax`` corrections). The solve policy then runs
the tier, among the predicted one and those of higher precision, with the least
measured cost per solve for the matrix's order and kind on this GPU (a cost table
calibrated by selector_train.py and stored with the weights): where refinement
does not pay, that is the plain fp64 solve. Features, inference, the training
forward/backward pass and the Adam update are the library's own CUDA kernels
(csrc/selector.cuh, C-ABI tsdx_cuda_selector_features_f64 / tsdx_cuda_mlp_* /
tsdx_cuda_adam_step); labels come from running the refinement kernel itself on
each tier (``label``). At solve time the refinement's residual check remains the
judge: a matrix whose predicted tier does not converge is re-solved by the plain
fp64 kernel in the same call, so a wrong prediction costs time, never accuracy.

No TinySolverDx counterpart (the reference has no GPU mixed-precision path).
torch tensors serve only as device buffers and for batching/shuffling indices.
"""
import numpy as np
import torch

from . import capi, device

TIERS = ("fp16", "bf16", "fp32", "fp64")
N_FEAT, N_HID, N_TIER = 24, 64, 4
N_PARAM = N_FEAT * N_HID + N_HID + N_HID * N_HID + N_HID + N_HID * N_TIER + N_TIER  # 6020


def _check(t, name, dtype):
    if not (t.is_cuda and t.is_contiguous()):
        raise ValueError(f"{name} must be a contiguous CUDA tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, not {t.dtype}")


def features(A, kind, stream=None):
    """(batch, 24) float32 features of the float64 CUDA stack A (batch, n, n).
    kind: 0 (SPD / Cholesky) or 1 (general / LU), or an int8 (batch,) tensor."""
    _check(A, "A", torch.float64)
    batch, n = A.shape[0], A.shape[-1]
    out = torch.empty(batch, N_FEAT, dtype=torch.float32, device=A.device)
    kt = kind if torch.is_tensor(kind) else None
    if kt is not None:
        _check(kt, "kind", torch.int8)
    capi.check(capi.call("tsdx_cuda_selector_features_f64", capi.ptr(A), n, batch, capi.ptr(kt),
                         0 if kt is not None else int(kind), capi.ptr(out), capi.stream_ptr(stream)),
               "selector features")
    return out


def label(A, b, spd, itmax=3, tol=1e-15, tiers=(0, 1, 2)):
    """Label = the first tier in ``tiers`` (lowest precision first) whose refinement converges
    within itmax corrections on (A, b); 3 (fp64) when none does. int8 CUDA tensor."""
    lab = torch.full((A.shape[0],), 3, dtype=torch.int8, device=A.device)
    for t in reversed(tiers):
        x = b.clone()
        _, status, _ = device.ir(A, x, spd, default_tier=t, itmax=itmax, tol=tol)
        lab = torch.where(status >= 0, torch.full_like(lab, t), lab)
    return lab


class Selector:
    """The network's parameters (flat float32, layout of csrc/selector.cuh), the
    feature normaliser (mu, 1/sd) and Adam state, all on one CUDA device."""

    def __init__(self, seed=0, device="cuda"):
        self.device = torch.device(device)
        rng = np.random.default_rng(seed)

        def he(fan_in, shape):
            lim = np.sqrt(6.0 / fan_in)
            return rng.uniform(-lim, lim, shape).astype(np.float32).ravel()

        p = np.concatenate([he(N_FEAT, (N_FEAT, N_HID)), np.zeros(N_HID, np.float32),
                            he(N_HID, (N_HID, N_HID)), np.zeros(N_HID, np.float32),
                            he(N_HID, (N_HID, N_TIER)), np.zeros(N_TIER, np.float32)])
        assert p.size == N_PARAM
        self.params = torch.from_numpy(p).to(self.device)
        self.norm = torch.cat([torch.zeros(N_FEAT), torch.ones(N_FEAT)]).to(self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.step = 0
        self.cost = None    # (len(cost_n), 2 kinds, 4 tiers) ns per solve, or None
        self.cost_n = None

    # a predicted tier t means t converges; these tiers are expected to converge too
    # (fp16 carries more precision than bf16 once the matrix is scaled into range)
    CANDIDATES = {0: (0, 2, 3), 1: (1, 0, 2, 3), 2: (2, 3), 3: (3,)}

    # a lower tier runs only when its cost (features and network included) is below
    # this fraction of the fp64 cost: the table is measured at kappa <= 10, where every
    # tier converges in few corrections, and a routed batch takes one more launch
    ROUTE_MARGIN = 0.9

    def policy_lut(self, n, spd):
        """int8 (4,) map from predicted tier to the tier to run for order n and kind."""
        lut = np.arange(4, dtype=np.int8)
        if self.cost is not None:
            i = int(np.argmin(np.abs(np.asarray(self.cost_n) - n)))
            c = np.array(self.cost[i, 0 if spd else 1], dtype=np.float64)
            c[:3] = np.where(c[:3] <= self.ROUTE_MARGIN * c[3], c[:3], np.inf)
            for t, cand in self.CANDIDATES.items():
                lut[t] = min(cand, key=lambda u: c[u])
        return lut

    def policy(self, pred, n, spd):
        lut = torch.from_numpy(self.policy_lut(n, spd)).to(pred.device)
        return lut[pred.long()]

    # ---------------------------------------------------------------- inference
    def fit_normalizer(self, X):
        mu = X.mean(0)
        sd = X.std(0).clamp_min(1e-3)
        self.norm = torch.cat([mu, 1.0 / sd]).float().contiguous()

    def forward(self, X, stream=None):
        """(logits (batch, 4) float32, predicted tier (batch,) int8)."""
        _check(X, "X", torch.float32)
        B = X.shape[0]
        logits = torch.empty(B, N_TIER, dtype=torch.float32, device=X.device)
        tier = torch.empty(B, dtype=torch.int8, device=X.device)
        capi.check(capi.call("tsdx_cuda_mlp_forward", capi.ptr(self.params), capi.ptr(self.norm), capi.ptr(X), B,
                             capi.ptr(logits), capi.ptr(tier), capi.stream_ptr(stream)), "mlp forward")
        return logits, tier

    def predict(self, X):
        return self.forward(X)[1]

    # ----------------------------------------------------------------- training
    def loss_grad(self, X, y, class_weight=None, scratch=None):
        """Gradient (N_PARAM,) and loss of sum_s w_{y_s} CE_s / batch on the device."""
        _check(X, "X", torch.float32)
        _check(y, "y", torch.int8)
        B = X.shape[0]
        need = int(capi.call("tsdx_cuda_mlp_scratch_bytes", B))
        if scratch is None or scratch.numel() < need:
            scratch = torch.empty(need, dtype=torch.uint8, device=X.device)
        grad = torch.empty(N_PARAM, dtype=torch.float32, device=X.device)
        loss = torch.empty(1, dtype=torch.float32, device=X.device)
        cw = None if class_weight is None else torch.as_tensor(class_weight, dtype=torch.float32).to(X.device)
        capi.check(capi.call("tsdx_cuda_mlp_grad", capi.ptr(self.params), capi.ptr(self.norm), capi.ptr(X),
                             capi.ptr(y), capi.ptr(cw), B, capi.ptr(grad), capi.ptr(loss), capi.ptr(scratch),
                             scratch.numel(), capi.stream_ptr()), "mlp grad")
        return grad, loss

    def adam_step(self, grad, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        capi.check(capi.call("tsdx_cuda_adam_step", capi.ptr(self.params), capi.ptr(grad), capi.ptr(self.m),
                             capi.ptr(self.v), N_PARAM, float(lr), float(beta1), float(beta2), float(eps),
                             self.step, capi.stream_ptr()), "adam step")

    def fit(self, X, y, epochs=5, batch_size=4096, lr=3e-3, class_weight=None, seed=0):
        """Minibatch Adam over (X, y); fits the normaliser first. Returns the mean
        loss of each epoch."""
        self.fit_normalizer(X)
        g = torch.Generator(device=X.device)
        g.manual_seed(seed)
        N = X.shape[0]
        need = int(capi.call("tsdx_cuda_mlp_scratch_bytes", batch_size))
        scratch = torch.empty(need, dtype=torch.uint8, device=X.device)
        hist = []
        for _ in range(epochs):
            perm = torch.randperm(N, generator=g, device=X.device)
            tot = torch.zeros(1, device=X.device)
            nb = 0
            for i in range(0, N, batch_size):
                idx = perm[i:i + batch_size]
                grad, loss = self.loss_grad(X[idx].contiguous(), y[idx].contiguous(), class_weight, scratch)
                self.adam_step(grad, lr)
                tot += loss
                nb += 1
            hist.append(float(tot.item()) / max(nb, 1))
        return hist

    # --------------------------------------------------------------- persistence
    def state_dict(self):
        d = {"params": self.params.cpu().numpy(), "norm": self.norm.cpu().numpy()}
        if self.cost is not None:
            d["cost"] = np.asarray(self.cost)
            d["cost_n"] = np.asarray(self.cost_n)
        return d

    def load_state_dict(self, d):
        self.params = torch.as_tensor(np.asarray(d["params"], np.float32)).to(self.device).contiguous()
        self.norm = torch.as_tensor(np.asarray(d["norm"], np.float32)).to(self.device).contiguous()
        if "cost" in d:
            self.cost = np.asarray(d["cost"], np.float64)
            self.cost_n = np.asarray(d["cost_n"], np.int64)

    def save(self, path):
        np.savez(path, **self.state_dict())

    @classmethod
    def load(cls, path, device="cuda"):
        s = cls(device=device)
        with np.load(path) as d:
            s.load_state_dict(d)
        return s

    # -------------------------------------------------------------------- solve
    def solve(self, A, b, spd, itmax=3, tol=1e-15):
        """Predict the lowest converging tier per matrix, run the cheapest tier at or
        above it (policy_lut), refine, fall back to fp64 on a miss.
        A (batch, n, n) float64, b (batch, n) float64 overwritten by x.
        Returns (info, status, bwd, tier run)."""
        n = A.shape[-1]
        lut = self.policy_lut(n, spd)
        if (lut == 3).all():
            # no tier is cheaper than fp64 at this order on this GPU: skip the features
            # and the network, solve in plain fp64
            info, status, bwd = device.ir(A, b, spd, default_tier=3, itmax=itmax, tol=tol)
            return info, status, bwd, torch.full_like(status, 3, dtype=torch.int8)
        X = features(A, 0 if spd else 1)
        tier = torch.from_numpy(lut).to(A.device)[self.predict(X).long()].contiguous()
        info, status, bwd = device.ir(A, b, spd, tier=tier, itmax=itmax, tol=tol)
        return info, status, bwd, tier

    def solve_host(self, parts, itmax=3, tol=1e-15, chunk_bytes=96 << 20, slots=3):
        """``solve`` on batches held in host memory, with the copies overlapping the solves.

        parts: list of (A, b, spd): A (batch, n, n) and b (batch, n) contiguous float64
        CPU tensors, spd a bool; b is overwritten by x. Pin A and b
        (``tensor.pin_memory()``) for the copies to overlap. Every part is cut into
        chunks of about ``chunk_bytes`` of A, and chunk c runs on stream c % slots as
        host->device copy, ``solve``, device->host copy, so the copies of one chunk
        overlap the solves of its neighbours, across parts too. The device holds
        ``slots`` chunks at a time. Returns one (info, status, tier) triple of CPU
        tensors per part; synchronous."""
        outs, jobs = [], []
        for A, b, spd in parts:
            for t, nm in ((A, "A"), (b, "b")):
                if t.is_cuda or not t.is_contiguous() or t.dtype != torch.float64:
                    raise ValueError(f"{nm} must be a contiguous float64 CPU tensor")
            if A.dim() != 3 or A.shape[1] != A.shape[2] or tuple(b.shape) != (A.shape[0], A.shape[1]):
                raise ValueError("A must be (batch, n, n) and b (batch, n)")
            batch, n = A.shape[0], A.shape[-1]
            pin = A.is_pinned()
            out = (torch.empty(batch, dtype=torch.int32, pin_memory=pin),
                   torch.empty(batch, dtype=torch.int32, pin_memory=pin),
                   torch.empty(batch, dtype=torch.int8, pin_memory=pin))
            outs.append(out)
            per = max(1, chunk_bytes // (n * n * 8))
            jobs += [(A, b, bool(spd), n, i0, min(batch, i0 + per), out) for i0 in range(0, batch, per)]
        if not jobs:
            return outs
        cur = torch.cuda.current_stream(self.device)
        mA = max((i1 - i0) * n * n for _, _, _, n, i0, i1, _ in jobs)
        mx = max((i1 - i0) * n for _, _, _, n, i0, i1, _ in jobs)
        bufA = [torch.empty(mA, dtype=torch.float64, device=self.device) for _ in range(slots)]
        bufx = [torch.empty(mx, dtype=torch.float64, device=self.device) for _ in range(slots)]
        streams = [torch.cuda.Stream(self.device) for _ in range(slots)]
        for st in streams:
            st.wait_stream(cur)  # the slot buffers were allocated on the current stream
        try:
            for c, (A, b, spd, n, i0, i1, (info, status, tier)) in enumerate(jobs):
                k, cnt = c % slots, i1 - i0
                # slot k's buffers are reused by chunk c + slots on the same stream, after
                # this chunk's copies back; the solve's own temporaries live on that stream too
                with torch.cuda.stream(streams[k]):
                    dA = bufA[k][:cnt * n * n].view(cnt, n, n)
                    dx = bufx[k][:cnt * n].view(cnt, n)
                    dA.copy_(A[i0:i1], non_blocking=True)
                    dx.copy_(b[i0:i1], non_blocking=True)
                    inf, stt, _, tr = self.solve(dA, dx, spd, itmax=itmax, tol=tol)
                    b[i0:i1].copy_(dx, non_blocking=True)
                    info[i0:i1].copy_(inf, non_blocking=True)
                    status[i0:i1].copy_(stt, non_blocking=True)
                    tier[i0:i1].copy_(tr, non_blocking=True)
        finally:
            # also on an error: no copy into the caller's buffers outlives the call
            for st in streams:
                st.synchronize()
        return outs
