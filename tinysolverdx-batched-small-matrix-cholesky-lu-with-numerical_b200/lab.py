"""Numerical error lab on the GPU: backward error against condition number and
size, per precision tier, written as CSV and a markdown table.

    python lab.py --out DIR [--quick] [--trials 4096] [--seed 0]

The reference's lab (python/tinysolverdx/lab.py:36-200) sweeps its CPU precisions
on the same inputs and judges them against long-double ground truth. This one
sweeps the GPU tiers on the same inputs, Cholesky (SPD) and LU (general), built
with the benchmark construction (matrices.torch_stack):
  * mixed precision: fp16, bf16 and fp32 factorizations with fp64 refinement
    (at most 3 corrections, tolerance 1e-15, fp64 fallback on a miss), reporting
    the fraction refined without fallback, the median number of corrections and
    the backward error of the returned x;
  * plain fp64 on the same inputs;
  * the reference's emulated per-operation-rounded fp16 / bf16 factorizations
    (run on the GPU, bit-identical to the CPU path), reporting the factorization
    backward error ||P A - L U|| / ||A|| or ||A - L L^T|| / ||A||.
Errors are measured on the device in double-double arithmetic (the reference's
runtime.cpp:194-242 metrics, which the reference evaluates in long double).
Plots are left out (no plotting library is assumed); the markdown table carries
the numbers.
"""
import argparse
import csv
import importlib
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent))
PKG = HERE.name
TIERS = ("fp16", "bf16", "fp32", "fp64")


def _med(t):
    t = t[t == t]
    return float(t.median().item()) if t.numel() else float("nan")


def _max(t):
    t = t[t == t]
    return float(t.max().item()) if t.numel() else float("nan")


def mixed_rows(n, kappa, trials, seed, device="cuda"):
    import torch
    M = importlib.import_module(PKG + ".matrices")
    dev = importlib.import_module(PKG + ".device")
    rows = []
    for spd in (True, False):
        A = M.torch_stack("spd" if spd else "general", n, trials, kappa, kappa, seed, device=device).contiguous()
        g = torch.Generator(device=device)
        g.manual_seed(seed + 1)
        b = torch.randn(trials, n, generator=g, device=device, dtype=torch.float64)
        for t, name in enumerate(TIERS):
            x = b.clone()
            info, status, _ = dev.ir(A, x, spd, default_tier=t)
            be = dev.solve_backward_error(A, x, b)
            refined = (status >= 0) if t < 3 else torch.zeros_like(status, dtype=torch.bool)
            steps = status[refined].float()
            rows.append({"section": "mixed", "kind": "cholesky" if spd else "lu", "n": n, "kappa": kappa,
                         "tier": name, "trials": trials,
                         "refined_frac": float(refined.float().mean().item()) if t < 3 else float("nan"),
                         "steps_med": _med(steps) if steps.numel() else float("nan"),
                         "backward_med": _med(be), "backward_max": _max(be)})
    return rows


def emulated_rows(n, kappa, trials, seed):
    import torch
    tsdx = importlib.import_module(PKG)
    M = importlib.import_module(PKG + ".matrices")
    dev = importlib.import_module(PKG + ".device")
    rng = np.random.default_rng(seed)
    rows = []
    for prec in ("fp16", "bf16"):
        for spd in (True, False):
            A = tsdx.round_to((M.spd if spd else M.general)(rng, trials, n, kappa), prec)
            Ad = torch.from_numpy(A).cuda()
            if spd:
                L, info = tsdx.cholesky(A, precision=prec, backend="cuda")
                be = dev.chol_backward_error(Ad, torch.from_numpy(np.ascontiguousarray(L, np.float64)).cuda())
            else:
                LU, piv, info = tsdx.lu(A, precision=prec, backend="cuda")
                be = dev.lu_backward_error(Ad, torch.from_numpy(np.ascontiguousarray(LU, np.float64)).cuda(),
                                           torch.from_numpy(piv.astype(np.int32)).cuda())
            ok = torch.from_numpy(info == 0).cuda() & torch.isfinite(be)
            rows.append({"section": "emulated", "kind": "cholesky" if spd else "lu", "n": n, "kappa": kappa,
                         "tier": prec, "trials": trials, "refined_frac": float("nan"), "steps_med": float("nan"),
                         "fail_frac": float(1 - ok.float().mean().item()),
                         "backward_med": _med(be[ok]), "backward_max": _max(be[ok])})
    return rows


def fmt(v):
    return "—" if v != v else (f"{v:.2e}" if abs(v) < 1e-2 or abs(v) >= 1e3 else f"{v:.3g}")


def write(out, rows):
    out.mkdir(parents=True, exist_ok=True)
    keys = ["section", "kind", "n", "kappa", "tier", "trials", "refined_frac", "steps_med", "fail_frac",
            "backward_med", "backward_max"]
    with open(out / "gpu_lab.csv", "w", newline="") as f:
        w = csv.DictWriter(f, keys)
        w.writeheader()
        for r in rows:
            w.writerow({k: r.get(k, "") for k in keys})
    lines = ["# GPU error lab", "",
             "## Mixed precision + fp64 refinement (backward error of the returned x)", "",
             "| kind | n | kappa | tier | refined w/o fallback | median corrections | bwd median | bwd max |",
             "|---|---|---|---|---|---|---|---|"]
    for r in rows:
        if r["section"] == "mixed":
            lines.append(f"| {r['kind']} | {r['n']} | {r['kappa']:.0e} | {r['tier']} | {fmt(r['refined_frac'])} | "
                         f"{fmt(r['steps_med'])} | {fmt(r['backward_med'])} | {fmt(r['backward_max'])} |")
    lines += ["", "## Emulated per-operation-rounded formats (factorization backward error)", "",
              "| kind | n | kappa | format | failed | bwd median | bwd max |", "|---|---|---|---|---|---|---|"]
    for r in rows:
        if r["section"] == "emulated":
            lines.append(f"| {r['kind']} | {r['n']} | {r['kappa']:.0e} | {r['tier']} | {fmt(r['fail_frac'])} | "
                         f"{fmt(r['backward_med'])} | {fmt(r['backward_max'])} |")
    (out / "gpu_lab.md").write_text("\n".join(lines) + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default="lab_out")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--trials", type=int, default=4096)
    ap.add_argument("--quick", action="store_true", help="fewer sizes and trials")
    a = ap.parse_args(argv)
    sizes = (16, 64) if a.quick else (16, 32, 64)
    kappas = (1e1, 1e4, 1e8, 1e12) if a.quick else (1e1, 1e3, 1e6, 1e9, 1e12)
    trials = min(a.trials, 1024) if a.quick else a.trials
    rows = []
    for i, n in enumerate(sizes):
        for j, k in enumerate(kappas):
            rows += mixed_rows(n, k, trials, a.seed + 100 * i + j)
    for j, k in enumerate(kappas):
        rows += emulated_rows(16, k, 256 if not a.quick else 64, a.seed + 7 + j)
    write(pathlib.Path(a.out), rows)
    print((pathlib.Path(a.out) / "gpu_lab.md").read_text())


if __name__ == "__main__":
    main()
