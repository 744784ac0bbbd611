"""Train the precision-tier selector and write its weights (selector_weights.npz).

    python selector_train.py [--count 2000000] [--epochs 12] [--out selector_weights.npz]
    python selector_train.py --calibrate-only [--out selector_weights.npz]

Training set: ``count`` seeded synthetic matrices, n uniform over 8..64, half
symmetric positive definite (Cholesky) and half general (LU), condition number
log-uniform in [1e0, 1e14], built on the device with the same construction as
the benchmarks (matrices.torch_stack), one right-hand side N(0, 1). Each matrix
is labelled with the lowest-precision tier (in the order fp16, bf16, fp32, fp64)
whose refinement converges to a normwise backward error <= 1e-15 within 3
corrections, by running the refinement kernel itself on every tier. A cost table
(ns per solve of each tier, per order and kind, measured on this GPU) is stored
with the weights; the solve policy uses it to pick the cheapest tier at or above
the predicted one; --calibrate-only re-measures that table for the kernels
built now and keeps the trained network. Features, training forward/backward
and the Adam updates all run in the library's own kernels. The matrices are
generated and dropped group by group; only features and labels are kept.
"""
import argparse
import importlib
import json
import pathlib
import sys
import time

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
PKG = HERE.name
SIZES = tuple(range(8, 65))


def dataset(count, seed, device="cuda", sizes=SIZES, kappa=(1e0, 1e14), keep=False):
    """(X, y, groups): features and labels of ``count`` matrices in (n, kind) groups.
    With keep=True the groups also hold (A, b) for evaluation."""
    import torch
    M = importlib.import_module(PKG + ".matrices")
    sel = importlib.import_module(PKG + ".selector")
    rng = np.random.default_rng(seed)
    ns = rng.choice(sizes, count)
    kinds = rng.integers(0, 2, count)
    Xs, ys, groups = [], [], []
    gid = 0
    for n in sizes:
        for spd in (False, True):
            c = int(((ns == n) & (kinds == (0 if spd else 1))).sum())
            if c == 0:
                continue
            A = M.torch_stack("spd" if spd else "general", n, c, kappa[0], kappa[1], seed * 1000 + gid,
                              device=device).contiguous()
            g = torch.Generator(device=device)
            g.manual_seed(seed * 1000 + gid + 500)
            b = torch.randn(c, n, generator=g, device=device, dtype=torch.float64)
            X = sel.features(A, 0 if spd else 1)
            y = sel.label(A, b, spd)
            Xs.append(X)
            ys.append(y)
            groups.append({"n": int(n), "spd": spd, "count": c, "A": A if keep else None, "b": b if keep else None,
                           "X": X, "y": y})
            gid += 1
    return torch.cat(Xs), torch.cat(ys), groups


def calibrate(device="cuda", sizes=(8, 16, 24, 32, 40, 48, 56, 64), count=16384, reps=3, sel=None):
    """Measured ns per solve of each tier on well-conditioned matrices (kappa <= 10,
    where every tier converges): cost[size][kind (0 SPD, 1 general)][tier], tier 3 =
    the plain fp64 solve. The lower tiers include the selector's own pass (features
    and network forward) when ``sel`` is given. CUDA events, best of ``reps``."""
    import torch
    M = importlib.import_module(PKG + ".matrices")
    dev = importlib.import_module(PKG + ".device")
    selm = importlib.import_module(PKG + ".selector")
    cost = np.zeros((len(sizes), 2, 4))
    for i, n in enumerate(sizes):
        for kd, spd in ((0, True), (1, False)):
            A = M.torch_stack("spd" if spd else "general", n, count, 1.0, 10.0, 900 + i * 2 + kd,
                              device=device).contiguous()
            b = torch.randn(count, n, device=device, dtype=torch.float64)
            for t in range(4):
                best = float("inf")
                for _ in range(reps + 1):
                    x = b.clone()
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    dev.ir(A, x, spd, default_tier=t)
                    e1.record()
                    e1.synchronize()
                    best = min(best, e0.elapsed_time(e1))
                cost[i, kd, t] = best * 1e6 / count
            if sel is not None:
                best = float("inf")
                for _ in range(reps + 1):
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    sel.predict(selm.features(A, kd))
                    e1.record()
                    e1.synchronize()
                    best = min(best, e0.elapsed_time(e1))
                cost[i, kd, :3] += best * 1e6 / count
    return cost, np.asarray(sizes)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--count", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--out", default=str(HERE / "selector_weights.npz"))
    ap.add_argument("--calibrate-only", action="store_true",
                    help="keep the network in --out and re-measure only its cost table")
    a = ap.parse_args(argv)
    import torch
    sel = importlib.import_module(PKG + ".selector")
    if a.calibrate_only:
        s = sel.Selector.load(a.out)
        s.cost, s.cost_n = calibrate(sel=s)
        s.save(a.out)
        print(json.dumps({"out": a.out, "cost_ns_per_solve": {
            int(n): {"spd": [round(v, 1) for v in s.cost[i, 0]], "general": [round(v, 1) for v in s.cost[i, 1]]}
            for i, n in enumerate(s.cost_n)}}), flush=True)
        return
    t0 = time.time()
    X, y, _ = dataset(a.count, a.seed)
    counts = torch.bincount(y.long(), minlength=4).cpu().tolist()
    t1 = time.time()
    s = sel.Selector(seed=a.seed)
    hist = s.fit(X, y, epochs=a.epochs, batch_size=a.batch, lr=a.lr)
    torch.cuda.synchronize()
    t2 = time.time()
    acc = (s.predict(X) == y).float().mean().item()
    s.cost, s.cost_n = calibrate(sel=s)
    s.save(a.out)
    print(json.dumps({"count": a.count, "label_counts": dict(zip(sel.TIERS, counts)), "epochs": a.epochs,
                      "loss": [round(v, 4) for v in hist], "train_accuracy": round(acc, 4),
                      "data_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1), "out": a.out,
                      "cost_ns_per_solve": {int(n): {"spd": [round(v, 1) for v in s.cost[i, 0]],
                                                     "general": [round(v, 1) for v in s.cost[i, 1]]}
                                            for i, n in enumerate(s.cost_n)}}), flush=True)


if __name__ == "__main__":
    main()
