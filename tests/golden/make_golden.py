"""Generates tests/golden/golden.npz from the REFERENCE itself.

Run where the reference tree is present (it reads it; nothing else does):

    make -C oracle ref REF=/path/to/reference   # oracle/_ref/libtsdx_ref.so from its sources
    python tests/golden/make_golden.py /path/to/reference   (or TSDX_REFERENCE=/path/to/reference)

Inputs come from the reference's own generator (python/tinysolverdx/matrices.py,
imported by path) and the reference tests' fixtures (tests/cpp/test_solvers.cpp
make_spd / make_general shapes, the 2x2 pivot example, the info examples);
outputs come from the reference library compiled from its sources, so the
fixtures pin both the C restatement in oracle/ and the GPU path.
"""
import importlib.util
import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
from oracle.oracle import Oracle  # noqa: E402


def ref_matrices(ref_root):
    spec = importlib.util.spec_from_file_location(
        "ref_matrices", pathlib.Path(ref_root) / "python" / "tinysolverdx" / "matrices.py")
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def main(ref_root):
    M = ref_matrices(ref_root)
    R = Oracle("reference")
    out = {}
    sizes64 = [1, 2, 3, 5, 8, 16, 17, 24, 25, 32, 33, 64]
    sizes32 = [2, 5, 16, 17, 32, 64]
    batch = 3
    for dt, sizes in ((np.float64, sizes64), (np.float32, sizes32)):
        tag = "f64" if dt == np.float64 else "f32"
        for n in sizes:
            rng = np.random.default_rng(1000 + n)
            S = M.spd(rng, batch, n, 1e3).astype(dt)
            G = M.general(rng, batch, n, 1e4).astype(dt)
            if n >= 3:
                G[1, :, n // 2] = 0.0          # one zeroed column -> info > 0
            nrhs = 1 if n % 2 else 3
            B = rng.standard_normal((batch, n, nrhs)).astype(dt)
            L, info = R.cholesky(S, "auto")              # simd semantics
            Ls, infos = R.cholesky(S, "scalar")
            LU, piv, linfo = R.lu(G, "auto")
            X = R.cholesky_solve(L, B)
            Y = R.lu_solve(LU, piv, B)
            k = f"{tag}_n{n}"
            out.update({f"{k}_spd": S, f"{k}_gen": G, f"{k}_B": B,
                        f"{k}_L": L, f"{k}_info": info, f"{k}_Lscalar": Ls,
                        f"{k}_LU": LU, f"{k}_piv": piv, f"{k}_luinfo": linfo,
                        f"{k}_Xchol": X, f"{k}_Xlu": Y})
    # known-answer cases from tests/cpp/test_solvers.cpp
    out["kat_pivot2"] = np.array([[[0.0, 1.0], [1.0, 0.0]]])   # :143-155 -> piv [1, 1]
    rng = np.random.default_rng(7)
    Sn = M.spd(rng, 11, 5, 10.0)
    Sn[3, 2, 2] = -1.0                                          # :78-92 (info 3 expected > 0)
    Sn[9] = 0.0                                                 # zero matrix -> info 1
    out["kat_nonspd"] = Sn
    out["kat_nonspd_info"] = R.cholesky(Sn, "auto")[1]
    Gs = rng.standard_normal((9, 4, 4))
    Gs[4, 2] = Gs[4, 1]                                         # :157-171 duplicate rows
    Gs[6] = 0.0                                                 # zero matrix -> info 1
    out["kat_singular"] = Gs
    _, out["kat_singular_piv"], out["kat_singular_info"] = R.lu(Gs, "auto")
    # fp16 / bf16 rounding known answers (tests/cpp/test_precision.cpp:10-30)
    xs = np.array([1.0, 1 + 1 / 2048, 1 + 3 / 2048, 65504.0, 65520.0, 6.0e-8, 1.0e-9, -0.1,
                   1 + 1 / 256, 1 + 3 / 256, 3.14159265, 3.4e38], np.float32)
    out["round_x"] = xs
    out["round_fp16"] = np.array([R.round_fp16(x) for x in xs], np.float32)
    out["round_bf16"] = np.array([R.round_bf16(x) for x in xs], np.float32)
    # long-double metrics (runtime.cpp:194-260)
    rng = np.random.default_rng(5)
    A = M.general(rng, 6, 10, 1e4)
    b = rng.standard_normal((6, 10))
    LU, piv, _ = R.lu(A, "auto")
    x = R.lu_solve(LU, piv, b[..., None])[..., 0]
    out.update(metric_A=A, metric_b=b, metric_x=x,
               metric_lu_bwd=R.lu_backward_error(A, LU, piv),
               metric_solve_bwd=R.solve_backward_error(A, x, b),
               metric_solve_fwd=R.solve_forward_error(A, x, b),
               metric_xref=R.reference_solve(A, b))
    S = M.spd(rng, 6, 10, 1e4)
    Lc, _ = R.cholesky(S, "auto")
    out.update(metric_S=S, metric_chol_bwd=R.chol_backward_error(S, Lc))
    np.savez_compressed(HERE / "golden.npz", **out)
    print("wrote", HERE / "golden.npz", sum(v.nbytes for v in out.values()), "bytes raw")


if __name__ == "__main__":
    import os
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("TSDX_REFERENCE")
    if not root:
        sys.exit("usage: make_golden.py <reference source tree>  (or set TSDX_REFERENCE)")
    main(root)
