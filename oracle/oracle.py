"""ctypes front-end of the CPU checker (test infrastructure, never the product).

Two libraries sit behind the same numpy-level functions:

* ``Oracle(kind="port")`` loads ``oracle/liboracle.so``, the plain-C
  restatement of the reference arithmetic in ``tsdx_oracle.c``.
* ``Oracle(kind="reference")`` loads ``oracle/_ref/libtsdx_ref.so``, the
  reference library compiled from its own sources by ``oracle/Makefile``.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` import this module.
"""
import ctypes as C
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
PORT_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libtsdx_ref.so"

BACKENDS = {"auto": 0, "naive": 1, "scalar": 2, "simd": 3}
PRECISIONS = {"fp32": 0, "fp64": 1, "fp16": 2, "bf16": 3}

_P = C.c_void_p
_I64 = C.c_int64


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def build(reference=True):
    """Compile the checker libraries (make -C oracle)."""
    import subprocess
    target = "all" if reference else str(PORT_LIB)
    subprocess.run(["make", "-s", "-C", str(HERE), target], check=True)


def ref_available():
    return REF_LIB.exists()


class Oracle:
    """Batched CPU solver with the reference's numpy-facing semantics."""

    def __init__(self, kind="port"):
        self.kind = kind
        path = PORT_LIB if kind == "port" else REF_LIB
        if not path.exists():
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        self.lib = C.CDLL(str(path))
        self.pre = "orc_" if kind == "port" else "ref_"
        for s in ("f", "d"):
            for name, args in (
                ("cholesky_batched", [_P, C.c_int, _I64, _P, C.c_int]),
                ("lu_batched", [_P, C.c_int, _I64, _P, _P, C.c_int]),
                ("cholesky_solve_batched", [_P, C.c_int, _I64, _P, C.c_int]),
                ("lu_solve_batched", [_P, _P, C.c_int, _I64, _P, C.c_int]),
            ):
                fn = getattr(self.lib, f"{self.pre}{name}_{s}")
                fn.argtypes = args
        getattr(self.lib, self.pre + "chol_backward_error").argtypes = [_P, _P, C.c_int, _I64, _P]
        for name in ("solve_backward_error", "solve_forward_error"):
            getattr(self.lib, self.pre + name).argtypes = [_P, _P, _P, C.c_int, _I64, _P]
        getattr(self.lib, self.pre + "lu_backward_error").argtypes = [_P, _P, _P, C.c_int, _I64, _P]
        getattr(self.lib, self.pre + "reference_solve").argtypes = [_P, _P, C.c_int, _I64, _P]
        for r in ("round_fp16", "round_bf16"):
            fn = getattr(self.lib, self.pre + r)
            fn.argtypes = [C.c_float]
            fn.restype = C.c_float
        if kind == "reference":
            self.lib.ref_set_num_threads.argtypes = [C.c_int]
            for s in ("f", "d"):
                getattr(self.lib, f"ref_posv_batched_{s}").argtypes = [_P, C.c_int, _I64, _P, C.c_int, _P, C.c_int]
                getattr(self.lib, f"ref_gesv_batched_{s}").argtypes = [_P, C.c_int, _I64, _P, C.c_int, _P, _P, C.c_int]
                getattr(self.lib, f"ref_cholesky_{s}").argtypes = [C.c_int, _P, C.c_int, _I64, _P, C.c_int]
                getattr(self.lib, f"ref_lu_{s}").argtypes = [C.c_int, _P, C.c_int, _I64, _P, _P, C.c_int]
                getattr(self.lib, f"ref_cholesky_solve_{s}").argtypes = [C.c_int, _P, C.c_int, _I64, _P, C.c_int]
                getattr(self.lib, f"ref_lu_solve_{s}").argtypes = [C.c_int, _P, _P, C.c_int, _I64, _P, C.c_int]
                getattr(self.lib, f"ref_round_to_{s}").argtypes = [C.c_int, _P, _I64]
        else:
            self.lib.orc_emu_cholesky.argtypes = [C.c_int, _P, C.c_int, _I64, _P]
            self.lib.orc_emu_lu.argtypes = [C.c_int, _P, C.c_int, _I64, _P, _P]
            self.lib.orc_emu_cholesky_solve.argtypes = [C.c_int, _P, C.c_int, _I64, _P, C.c_int]
            self.lib.orc_emu_lu_solve.argtypes = [C.c_int, _P, _P, C.c_int, _I64, _P, C.c_int]
            self.lib.orc_round_to.argtypes = [C.c_int, _P, _I64]

    # -- helpers ---------------------------------------------------------------
    @staticmethod
    def _sfx(a):
        if a.dtype == np.float64:
            return "d"
        if a.dtype == np.float32:
            return "f"
        raise TypeError(f"unsupported dtype {a.dtype}")

    def _call(self, name, *args):
        r = getattr(self.lib, self.pre + name)(*args)
        if self.kind == "reference" and isinstance(r, int) and r != 0 and name.endswith(("_f", "_d")):
            raise RuntimeError(f"reference call {name} raised")
        return r

    def set_num_threads(self, n):
        if self.kind == "reference":
            self.lib.ref_set_num_threads(int(n))

    # -- typed batched API (batched.hpp:121-280) --------------------------------
    def cholesky(self, A, backend="auto"):
        """Returns (L, info) for a (batch, n, n) float32/float64 stack."""
        a = np.array(A, copy=True, order="C")
        batch, n = a.shape[0], a.shape[1]
        info = np.zeros(batch, np.int32)
        self._call(f"cholesky_batched_{self._sfx(a)}", _ptr(a), n, batch, _ptr(info), BACKENDS[backend])
        return a, info

    def lu(self, A, backend="auto"):
        a = np.array(A, copy=True, order="C")
        batch, n = a.shape[0], a.shape[1]
        piv = np.zeros((batch, n), np.int32)
        info = np.zeros(batch, np.int32)
        self._call(f"lu_batched_{self._sfx(a)}", _ptr(a), n, batch, _ptr(piv), _ptr(info), BACKENDS[backend])
        return a, piv, info

    def cholesky_solve(self, L, B):
        L = np.ascontiguousarray(L)
        x = np.array(B, copy=True, order="C", dtype=L.dtype)
        self._call(f"cholesky_solve_batched_{self._sfx(L)}", _ptr(L), L.shape[1], L.shape[0], _ptr(x), x.shape[2])
        return x

    def lu_solve(self, LU, piv, B):
        LU = np.ascontiguousarray(LU)
        piv = np.ascontiguousarray(piv, dtype=np.int32)
        x = np.array(B, copy=True, order="C", dtype=LU.dtype)
        self._call(f"lu_solve_batched_{self._sfx(LU)}", _ptr(LU), _ptr(piv), LU.shape[1], LU.shape[0], _ptr(x), x.shape[2])
        return x

    def posv(self, A, B, backend="auto"):
        L, info = self.cholesky(A, backend)
        return L, self.cholesky_solve(L, B), info

    def gesv(self, A, B, backend="auto"):
        LU, piv, info = self.lu(A, backend)
        return LU, piv, self.lu_solve(LU, piv, B), info

    # -- emulated fp16 / bf16 (runtime.cpp:95-141 with precision.hpp:71-97) -------
    def emu_cholesky(self, prec, A):
        a = np.array(A, copy=True, order="C", dtype=np.float64)
        info = np.zeros(a.shape[0], np.int32)
        if self.kind == "port":
            self.lib.orc_emu_cholesky(0 if prec == "fp16" else 1, _ptr(a), a.shape[1], a.shape[0], _ptr(info))
        else:
            self._call("cholesky_d", PRECISIONS[prec], _ptr(a), a.shape[1], a.shape[0], _ptr(info), 0)
        return a, info

    def emu_lu(self, prec, A):
        a = np.array(A, copy=True, order="C", dtype=np.float64)
        piv = np.zeros(a.shape[:2], np.int32)
        info = np.zeros(a.shape[0], np.int32)
        if self.kind == "port":
            self.lib.orc_emu_lu(0 if prec == "fp16" else 1, _ptr(a), a.shape[1], a.shape[0], _ptr(piv), _ptr(info))
        else:
            self._call("lu_d", PRECISIONS[prec], _ptr(a), a.shape[1], a.shape[0], _ptr(piv), _ptr(info), 0)
        return a, piv, info

    def emu_cholesky_solve(self, prec, L, B):
        L = np.ascontiguousarray(L, dtype=np.float64)
        x = np.array(B, copy=True, order="C", dtype=np.float64)
        if self.kind == "port":
            self.lib.orc_emu_cholesky_solve(0 if prec == "fp16" else 1, _ptr(L), L.shape[1], L.shape[0], _ptr(x), x.shape[2])
        else:
            self._call("cholesky_solve_d", PRECISIONS[prec], _ptr(L), L.shape[1], L.shape[0], _ptr(x), x.shape[2])
        return x

    def emu_lu_solve(self, prec, LU, piv, B):
        LU = np.ascontiguousarray(LU, dtype=np.float64)
        piv = np.ascontiguousarray(piv, dtype=np.int32)
        x = np.array(B, copy=True, order="C", dtype=np.float64)
        if self.kind == "port":
            self.lib.orc_emu_lu_solve(0 if prec == "fp16" else 1, _ptr(LU), _ptr(piv), LU.shape[1], LU.shape[0], _ptr(x), x.shape[2])
        else:
            self._call("lu_solve_d", PRECISIONS[prec], _ptr(LU), _ptr(piv), LU.shape[1], LU.shape[0], _ptr(x), x.shape[2])
        return x

    def round_to(self, x, prec):
        a = np.array(x, copy=True, order="C", dtype=np.float64)
        if self.kind == "port":
            self.lib.orc_round_to(PRECISIONS[prec], _ptr(a), a.size)
        else:
            self.lib.ref_round_to_d(PRECISIONS[prec], _ptr(a), a.size)
        return a

    def round_fp16(self, x):
        return getattr(self.lib, self.pre + "round_fp16")(float(x))

    def round_bf16(self, x):
        return getattr(self.lib, self.pre + "round_bf16")(float(x))

    # -- long-double ground truth and metrics (runtime.cpp:162-260) ---------------
    def _metric(self, name, A, X, Bv):
        A = np.ascontiguousarray(A, dtype=np.float64)
        X = np.ascontiguousarray(X, dtype=np.float64)
        Bv = np.ascontiguousarray(Bv, dtype=np.float64)
        out = np.zeros(A.shape[0])
        getattr(self.lib, self.pre + name)(_ptr(A), _ptr(X), _ptr(Bv), A.shape[1], A.shape[0], _ptr(out))
        return out

    def chol_backward_error(self, A, L):
        A = np.ascontiguousarray(A, dtype=np.float64)
        L = np.ascontiguousarray(L, dtype=np.float64)
        out = np.zeros(A.shape[0])
        getattr(self.lib, self.pre + "chol_backward_error")(_ptr(A), _ptr(L), A.shape[1], A.shape[0], _ptr(out))
        return out

    def lu_backward_error(self, A, LU, piv):
        A = np.ascontiguousarray(A, dtype=np.float64)
        LU = np.ascontiguousarray(LU, dtype=np.float64)
        piv = np.ascontiguousarray(piv, dtype=np.int32)
        out = np.zeros(A.shape[0])
        getattr(self.lib, self.pre + "lu_backward_error")(_ptr(A), _ptr(LU), _ptr(piv), A.shape[1], A.shape[0], _ptr(out))
        return out

    def solve_backward_error(self, A, x, b):
        return self._metric("solve_backward_error", A, x, b)

    def solve_forward_error(self, A, x, b):
        return self._metric("solve_forward_error", A, x, b)

    def reference_solve(self, A, b):
        A = np.ascontiguousarray(A, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        getattr(self.lib, self.pre + "reference_solve")(_ptr(A), _ptr(b), A.shape[1], A.shape[0], _ptr(x))
        return x
