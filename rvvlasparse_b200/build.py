"""Build recipe for the in-tree CUDA library ``lib/librvvla_b200.so``.

Every ``csrc/*.cu`` file is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) in parallel, ``csrc/*.cpp``
(host code: workload generators, the C++ drop-in layer) with the same nvcc
host compiler, and the objects are linked into one shared library with the
CUDA runtime linked statically.  Objects are rebuilt only when a source or
header is newer.  The drop-in C++ test program under ``dropin/`` is built by
``build_dropin_test``.

Usage: ``python -m rvvlasparse_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OBJ_DIR = os.path.join(PKG, "_build", "obj")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "librvvla_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _host_cxx() -> list[str]:
    # The system g++ links OpenMP correctly; some environments export a CXX
    # wrapper without libgomp.spec.
    return ["-ccbin", "/usr/bin/g++"] if os.path.exists("/usr/bin/g++") else []


def _common_flags() -> list[str]:
    return [
        "-O3",
        "-std=c++17",
        "-lineinfo",
        "--expt-relaxed-constexpr",
        "-Xcompiler",
        "-fPIC,-fopenmp,-Wno-unused-function",
        "-I" + INCLUDE,
        "-I" + CSRC,
    ]


def _headers() -> list[str]:
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(
        os.path.join(INCLUDE, "*.h")
    )


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _compile(src: str, verbose: bool) -> str:
    obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
    if not _stale(obj, [src] + _headers()):
        return obj
    cmd = [_nvcc()] + _host_cxx() + _common_flags()
    if src.endswith(".cu"):
        cmd += ARCH
    cmd += ["-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{res.stdout}\n{res.stderr}")
    return obj


def build(verbose: bool = False, jobs: int | None = None) -> str:
    """Compile and link ``librvvla_b200.so``; returns its path."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    os.makedirs(LIB_DIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    jobs = jobs or max(1, min(len(srcs), os.cpu_count() or 4))
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [_nvcc()] + _host_cxx() + ARCH + ["-shared", "-o", tmp] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, LIB)
    return LIB


def ptxas_report(src: str) -> str:
    """Register / spill / shared-memory report (-Xptxas -v) for one source."""
    cmd = [_nvcc()] + _host_cxx() + _common_flags() + ARCH + ["-Xptxas", "-v", "-c", src, "-o", os.devnull]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return res.stdout + res.stderr


if __name__ == "__main__":
    path = build(verbose="-v" in sys.argv)
    print(path)
