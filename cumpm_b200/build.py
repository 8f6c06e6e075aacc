"""In-tree build of the CUDA library and the Python extension.

Produces, next to this file:
  * ``libcumpm_b200.so`` -- the C ABI declared in ``include/cumpm_b200.h``
    (CUDA kernels for sm_100a + host driver), linked against cuFFT;
  * ``_cuMPM<ext>`` -- the pybind11 module bound on top of that C ABI
    (rpath ``$ORIGIN`` so the pair travels together).

Usage: ``python cumpm_b200/build.py`` (or ``build()`` from Python).
Objects are cached under ``cumpm_b200/_build`` and rebuilt when a source or
header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
LIB = os.path.join(HERE, "libcumpm_b200.so")

LIB_SOURCES = ["mpm_tables.cpp", "mpm_profile.cpp", "mpm_fft.cu", "mpm_field.cu", "mpm_poly.cu", "mpm_adjoint.cu",
               "mpm_krylov.cu", "mpm_solver.cpp", "mpm_capi.cpp", "mpm_noalloc.cu", "mpm_tune.cpp"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I" + CSRC, "-I" + INCLUDE] + ARCH


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


def module_path() -> str:
    return os.path.join(HERE, "_cuMPM" + _ext_suffix())


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(INCLUDE, "cumpm_b200.h"))
    return hs


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build command failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if verbose and (r.stdout or r.stderr):
        print(r.stdout + r.stderr, flush=True)


def _compile(src: str, verbose: bool, extra=()) -> str:
    os.makedirs(BUILD, exist_ok=True)
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + _headers()
    if _stale(obj, deps):
        cmd = [NVCC] + NVFLAGS + list(extra) + ["-x", "cu", "-c", src, "-o", obj]
        _run(cmd, verbose)
    return obj


def build(verbose: bool = False) -> None:
    srcs = [os.path.join(CSRC, s) for s in LIB_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", LIB] + objs + ["-lcufft", "-lcudart"], verbose)
    # python extension (host-only C++; links the C ABI library)
    import pybind11

    py_inc = sysconfig.get_paths()["include"]
    src = os.path.join(CSRC, "mpm_pybind.cpp")
    mod = module_path()
    if _stale(mod, [src, LIB, os.path.join(INCLUDE, "cumpm_b200.h")]):
        cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden", "-I" + pybind11.get_include(),
               "-I" + py_inc, "-I" + INCLUDE, src, "-o", mod, "-L" + HERE, "-lcumpm_b200", "-Wl,-rpath,$ORIGIN"]
        _run(cmd, verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print("built", LIB, module_path())
