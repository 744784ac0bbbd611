"""Builds the sm_100a solver library and the pybind11 ``_core`` module in-tree.

    python <package>/build.py [--jobs N] [--force]

Outputs (git-ignored, shipped with the source tree to the GPU host):
  _lib/libtsdx_cuda.so   C-ABI of include/tsdx_cuda.h (nvcc, -arch sm_100a)
  _core*.so              pybind11 module mirroring TinySolverDx's ``_core``

nvcc cross-compiles without a GPU, so this runs on any machine with CUDA 12.9.
Objects are rebuilt only when a source or header is newer than the object.
"""
import argparse
import concurrent.futures as cf
import os
import pathlib
import re
import subprocess
import sys
import sysconfig

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OUT = PKG / "_lib"
OBJ = PKG / "_build"
LIB = OUT / "libtsdx_cuda.so"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                  "-I" + str(CSRC), "-I" + str(ROOT / "include")]
CUDA_SOURCES = ["capi.cu", "k_lu_f32.cu", "k_lu_f64.cu", "k_chol_f32.cu", "k_chol_f64.cu", "k_ir.cu", "k_stream_f32.cu", "k_stream_f64.cu", "k_stream_noalloc.cu", "k_selector.cu", "k_metrics.cu", "k_emu.cu"]


def _deps(path, seen=None):
    """The file and every local header it includes, transitively (#include "...")."""
    seen = set() if seen is None else seen
    path = path.resolve()
    if path in seen or not path.exists():
        return seen
    seen.add(path)
    for m in re.finditer(r'^\s*#\s*include\s+"([^"]+)"', path.read_text(), re.M):
        _deps(path.parent / m.group(1), seen)
    return seen


def _compile(src, force):
    obj = OBJ / (pathlib.Path(src).stem + ".o")
    s = CSRC / src
    if not force and obj.exists() and obj.stat().st_mtime >= max(d.stat().st_mtime for d in _deps(s)):
        return obj, None
    cmd = [NVCC] + NVFLAGS + ["-c", str(s), "-o", str(obj)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"{' '.join(cmd)}\n{r.stdout}\n{r.stderr}"
    return obj, None


def build_cuda(jobs=None, force=False):
    OBJ.mkdir(exist_ok=True)
    OUT.mkdir(exist_ok=True)
    jobs = jobs or max(1, os.cpu_count() or 1)
    with cf.ThreadPoolExecutor(jobs) as ex:
        res = list(ex.map(lambda s: _compile(s, force), CUDA_SOURCES))
    errs = [e for _, e in res if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [str(o) for o, _ in res]
    if force or not LIB.exists() or LIB.stat().st_mtime < max(pathlib.Path(o).stat().st_mtime for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", str(LIB)] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return LIB


def build_core(force=False):
    """pybind11 ``_core`` linking libtsdx_cuda.so (rpath $ORIGIN/_lib)."""
    import pybind11
    src = CSRC / "bindings.cpp"
    if not src.exists():
        return None
    suffix = sysconfig.get_config_var("EXT_SUFFIX")
    out = PKG / ("_core" + suffix)
    deps = [src, CSRC / "host_api.hpp", ROOT / "include" / "tsdx_cuda.h", LIB, pathlib.Path(__file__)]
    if not force and out.exists() and out.stat().st_mtime >= max(d.stat().st_mtime for d in deps if d.exists()):
        return out
    cxx = "/usr/bin/g++"
    cmd = [cxx, "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"],
           "-I" + str(CSRC), "-I" + str(ROOT / "include"),
           str(src), "-o", str(out), "-L" + str(OUT), "-ltsdx_cuda", "-Wl,-rpath,$ORIGIN/_lib"]
    subprocess.run(cmd, check=True)
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args(argv)
    print(build_cuda(a.jobs, a.force))
    print(build_core(a.force))


if __name__ == "__main__":
    sys.exit(main())
