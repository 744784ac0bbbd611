"""ctypes binding of the C-ABI in include/tsdx_cuda.h (the drop-in boundary).

This is how Python reaches the sm_100a kernels without going through the
pybind11 ``_core`` module; the test-suite and the benchmark use it with torch
CUDA tensors (device-pointer API) and with pinned numpy/torch host buffers
(host-pointer API). Loading fails loudly if ``_lib/libtsdx_cuda.so`` has not
been built: there is no CPU fallback.
"""
import ctypes as C
import pathlib

PKG = pathlib.Path(__file__).resolve().parent
LIB_PATH = PKG / "_lib" / "libtsdx_cuda.so"

TSDX_OK = 0
TSDX_ERR_N = -1
TSDX_ERR_BATCH = -2
TSDX_ERR_NULL = -3
TSDX_ERR_NRHS = -4
TSDX_ERR_CUDA = -5
TSDX_ERR_NODEV = -6
TSDX_ERR_TOO_LARGE = -7

_P, _I, _I64 = C.c_void_p, C.c_int, C.c_int64

# name -> argtypes (every function returns int)
SIGNATURES = {}
for _s in ("f32", "f64"):
    SIGNATURES.update({
        f"tsdx_cuda_potrf_{_s}": [_P, _I, _I64, _P, _P],
        f"tsdx_cuda_getrf_{_s}": [_P, _I, _I64, _P, _P, _P],
        f"tsdx_cuda_potrs_{_s}": [_P, _I, _I64, _P, _I, _P],
        f"tsdx_cuda_getrs_{_s}": [_P, _P, _I, _I64, _P, _I, _P],
        f"tsdx_cuda_posv_{_s}": [_P, _I, _I64, _P, _I, _P, _P],
        f"tsdx_cuda_gesv_{_s}": [_P, _I, _I64, _P, _I, _P, _P, _P],
        f"tsdx_cuda_cholesky_batched_host_{_s}": [_P, _I, _I64, _P],
        f"tsdx_cuda_lu_batched_host_{_s}": [_P, _I, _I64, _P, _P],
        f"tsdx_cuda_cholesky_solve_batched_host_{_s}": [_P, _I, _I64, _P, _I],
        f"tsdx_cuda_lu_solve_batched_host_{_s}": [_P, _P, _I, _I64, _P, _I],
        f"tsdx_cuda_posv_batched_host_{_s}": [_P, _I, _I64, _P, _I, _P],
        f"tsdx_cuda_gesv_batched_host_{_s}": [_P, _I, _I64, _P, _I, _P, _P],
        f"tsdx_cuda_gesv_solve_host_{_s}": [_P, _I, _I64, _P, _I, _P],
        f"tsdx_cuda_posv_solve_host_{_s}": [_P, _I, _I64, _P, _I, _P],
    })
SIGNATURES.update({"tsdx_cuda_available": [], "tsdx_cuda_launch_count": [],
                   "tsdx_internal_div_check_f64": [_P, _P, _P, _P, _I64, _P],
                   "tsdx_internal_div_check_f32": [_P, _P, _P, _P, _I64, _P],
                   "tsdx_cuda_gesv_ir_f64": [_P, _I, _I64, _P, _P, _I, _I, C.c_double, _P, _P, _P, _P],
                   "tsdx_cuda_posv_ir_f64": [_P, _I, _I64, _P, _P, _I, _I, C.c_double, _P, _P, _P, _P],
                   "tsdx_cuda_stream_scratch_bytes": [_I64],
                   "tsdx_cuda_solve_stream_f32": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _I, C.c_uint, _P, _I64, _P],
                   "tsdx_cuda_solve_stream_f64": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _I, C.c_uint, _P, _I64, _P],
                   "tsdx_cuda_solve_stream_noalloc_f32": [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I64, _I, C.c_uint, _P],
                   "tsdx_cuda_solve_stream_host_f32": [_P, _P, _P, _P, _P, _P, _P, _I64, _I, C.c_uint],
                   "tsdx_cuda_solve_stream_host_f64": [_P, _P, _P, _P, _P, _P, _P, _I64, _I, C.c_uint],
                   "tsdx_cuda_emu_factor_host": [_I, _I, _P, _I, _I64, _P, _P],
                   "tsdx_cuda_emu_solve_host": [_I, _I, _P, _P, _I, _I64, _P, _I],
                   "tsdx_cuda_solve_backward_error_f64": [_P, _P, _P, _I, _I64, _P, _P],
                   "tsdx_cuda_lu_backward_error_f64": [_P, _P, _P, _I, _I64, _P, _P],
                   "tsdx_cuda_chol_backward_error_f64": [_P, _P, _I, _I64, _P, _P],
                   "tsdx_cuda_selector_features_f64": [_P, _I, _I64, _P, _I, _P, _P],
                   "tsdx_cuda_mlp_forward": [_P, _P, _P, _I64, _P, _P, _P],
                   "tsdx_cuda_mlp_scratch_bytes": [_I64],
                   "tsdx_cuda_mlp_grad": [_P, _P, _P, _P, _P, _I64, _P, _P, _P, _I64, _P],
                   "tsdx_cuda_adam_step": [_P, _P, _P, _P, _I64, C.c_float, C.c_float, C.c_float, C.c_float, _I,
                                           _P]})

_lib = None


def lib():
    """The loaded library (raises if it is not built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is not built; run build.py (no CPU fallback exists)")
        L = C.CDLL(str(LIB_PATH))
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = C.c_int64 if name in ("tsdx_cuda_launch_count", "tsdx_cuda_stream_scratch_bytes",
                                               "tsdx_cuda_mlp_scratch_bytes") else C.c_int
        L.tsdx_cuda_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def last_error():
    return lib().tsdx_cuda_last_error().decode()


def launch_count():
    return int(lib().tsdx_cuda_launch_count())


def check(rc, what=""):
    if rc != TSDX_OK:
        msg = {TSDX_ERR_N: "matrix size n outside supported range [1, 64]", TSDX_ERR_BATCH: "negative batch",
               TSDX_ERR_NULL: "null or misaligned pointer", TSDX_ERR_NRHS: "negative nrhs",
               TSDX_ERR_NODEV: "no CUDA device"}.get(rc)
        if rc in (TSDX_ERR_CUDA, TSDX_ERR_TOO_LARGE):
            if rc == TSDX_ERR_TOO_LARGE:
                raise ValueError(f"{what}: {last_error()}")
            raise RuntimeError(f"{what}: CUDA error: {last_error()}")
        if msg is None:
            raise RuntimeError(f"{what}: error {rc}")
        raise ValueError(f"{what}: {msg}")
    return rc


def call(name, *args):
    return getattr(lib(), name)(*args)


def ptr(t):
    """Raw data pointer of a torch tensor / numpy array (None -> NULL)."""
    if t is None:
        return None
    if hasattr(t, "data_ptr"):
        return C.c_void_p(t.data_ptr())
    return t.ctypes.data_as(C.c_void_p)


def sfx(dtype):
    s = str(dtype)
    if "float64" in s or "double" in s:
        return "f64"
    if "float32" in s:
        return "f32"
    raise TypeError(f"unsupported dtype {dtype}; use float32/float64")


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


# ---- device-tensor API (torch CUDA tensors, in place, stream-ordered) ----------
def potrf(A, info=None, stream=None):
    batch, n = A.shape[0], A.shape[-1]
    return check(call(f"tsdx_cuda_potrf_{sfx(A.dtype)}", ptr(A), n, batch, ptr(info), stream_ptr(stream)), "potrf")


def getrf(A, piv, info=None, stream=None):
    batch, n = A.shape[0], A.shape[-1]
    return check(call(f"tsdx_cuda_getrf_{sfx(A.dtype)}", ptr(A), n, batch, ptr(piv), ptr(info), stream_ptr(stream)), "getrf")


def potrs(L, B, stream=None):
    batch, n = L.shape[0], L.shape[-1]
    return check(call(f"tsdx_cuda_potrs_{sfx(L.dtype)}", ptr(L), n, batch, ptr(B), B.shape[-1], stream_ptr(stream)), "potrs")


def getrs(LU, piv, B, stream=None):
    batch, n = LU.shape[0], LU.shape[-1]
    return check(call(f"tsdx_cuda_getrs_{sfx(LU.dtype)}", ptr(LU), ptr(piv), n, batch, ptr(B), B.shape[-1], stream_ptr(stream)), "getrs")


def posv(A, B, info=None, stream=None):
    batch, n = A.shape[0], A.shape[-1]
    return check(call(f"tsdx_cuda_posv_{sfx(A.dtype)}", ptr(A), n, batch, ptr(B), B.shape[-1], ptr(info), stream_ptr(stream)), "posv")


def gesv(A, B, piv, info=None, stream=None):
    batch, n = A.shape[0], A.shape[-1]
    return check(call(f"tsdx_cuda_gesv_{sfx(A.dtype)}", ptr(A), n, batch, ptr(B), B.shape[-1], ptr(piv), ptr(info), stream_ptr(stream)), "gesv")
