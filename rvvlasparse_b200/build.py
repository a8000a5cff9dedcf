"""Build recipe for the in-tree CUDA library ``lib/librvvla_b200.so``.

Every ``csrc/*.cu`` file is compiled by nvcc for sm_100a only
(``-gencode arch=compute_100a,code=sm_100a``) in parallel, ``csrc/*.cpp``
(host code: workload generators, the VNEC/LAV host builders) with the same
nvcc host compiler, and the objects are linked into one shared library with
the CUDA runtime linked statically.  Objects are rebuilt only when a source or
header is newer.  ``build_dropin`` then compiles the C++ drop-in
(``dropin/dropin.cpp`` -> ``lib/librvvla_dropin.so``, the reference's C++ API
over the C ABI) and its test program (``_build/test_dropin``).

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


DROPIN = os.path.join(PKG, "dropin")
DROPIN_LIB = os.path.join(LIB_DIR, "librvvla_dropin.so")
DROPIN_TEST = os.path.join(PKG, "_build", "test_dropin")
DROPIN_BENCH = os.path.join(PKG, "_build", "bench_dropin")


def build_dropin(verbose: bool = False) -> str:
    """Compile the C++ drop-in library, its test program and the bench's
    end-to-end harness (host code only, linked against ``librvvla_b200.so``);
    returns the library path."""
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (shutil.which("g++") or "g++")
    inc = ["-I" + INCLUDE, "-I" + os.path.join(DROPIN, "include")]
    hdrs = glob.glob(os.path.join(DROPIN, "include", "*.h")) + [os.path.join(INCLUDE, "rvvla.h")]
    steps = [
        (DROPIN_LIB, [os.path.join(DROPIN, "dropin.cpp")],
         [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall"] + inc + [os.path.join(DROPIN, "dropin.cpp"),
          "-L" + LIB_DIR, "-lrvvla_b200", "-Wl,-rpath,$ORIGIN", "-o"]),
        (DROPIN_TEST, [os.path.join(DROPIN, "test_dropin.cpp"), DROPIN_LIB],
         [cxx, "-std=c++17", "-O2", "-Wall"] + inc + [os.path.join(DROPIN, "test_dropin.cpp"), "-L" + LIB_DIR,
          "-lrvvla_dropin", "-lrvvla_b200", "-Wl,-rpath,$ORIGIN/../lib", "-o"]),
        (DROPIN_BENCH, [os.path.join(DROPIN, "bench_dropin.cpp"), DROPIN_LIB],
         [cxx, "-std=c++17", "-O2", "-Wall"] + inc + [os.path.join(DROPIN, "bench_dropin.cpp"), "-L" + LIB_DIR,
          "-lrvvla_dropin", "-lrvvla_b200", "-Wl,-rpath,$ORIGIN/../lib", "-o"]),
    ]
    os.makedirs(os.path.dirname(DROPIN_TEST), exist_ok=True)
    for target, srcs, cmd in steps:
        if not _stale(target, srcs + hdrs + [LIB]):
            continue
        tmp = target + ".tmp"
        cmd = cmd + [tmp]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"drop-in build failed ({os.path.basename(target)}):\n{res.stdout}\n{res.stderr}")
        os.replace(tmp, target)
    return DROPIN_LIB


def ptxas_report(src: str) -> str:
    """Register / spill / shared-memory report (-Xptxas -v) for one source."""
    cmd = [_nvcc()] + _host_cxx() + _common_flags() + ARCH + ["-Xptxas", "-v", "-c", src, "-o", os.devnull]
    res = subprocess.run(cmd, capture_output=True, text=True)
    return res.stdout + res.stderr


if __name__ == "__main__":
    path = build(verbose="-v" in sys.argv)
    build_dropin(verbose="-v" in sys.argv)
    print(path)
