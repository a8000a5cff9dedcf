"""Measuring autotuner for the single-matrix formats (no reference counterpart).

``tune(fmt, A, ...)`` runs the library's tuner (``rvvla_autotune`` in the C
ABI): every candidate parameter set is built on the GPU, timed with CUDA
events (one untimed call, best of ``iters``), and the fastest parameters come
back with the table of all timings.  Candidates:

* ``csr5``  sigma in {8, 16, 24, 32} (omega is fixed to a warp, 32);
* ``sell``  C = 32 (a warp per slice) with sigma in {32, 256, 1024, 8192};
* ``hcsr``  square blocks R = C in {512, 1024, 2000, 4000, 8192},
  R in {1000, 2000, 4000} with C = 65536, and C = 65536 with R making the
  block rows 2, 3 or 4 whole waves of two CTAs per SM, p = 2;
* ``vhcc``  threads in {nnz/4096, nnz/2048, nnz/1024} (vectors of 32);
* ``cvr``   ranges of {8192, 32768, 131072} nonzeros;
* ``lav``   segment_len in {40000, n/4, n} (SIMD_Lanes 8, T 0.2).

The batched form has its own tuner in the library (``rvvla_batched_autotune``).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _capi
from . import formats as F

_CLASS = {"csr5": F.spMtxCSR5, "sell": F.spMtxSELL_C_Sigma, "hcsr": F.spMtxHCSR, "vhcc": F.spMtxVHCC,
          "cvr": F.spMtxCVR, "lav": F.spMtxLAV}
_FMT = {"hcsr": _capi.RVVLA_FMT_HCSR, "sell": _capi.RVVLA_FMT_SELL, "csr5": _capi.RVVLA_FMT_CSR5,
        "lav": _capi.RVVLA_FMT_LAV, "vhcc": _capi.RVVLA_FMT_VHCC, "cvr": _capi.RVVLA_FMT_CVR}


def _params(fmt: str, t: _capi.rvvla_tune_params) -> dict:
    """The convertParams keys of one tuned parameter set."""
    if fmt == "hcsr":
        return dict(R=int(t.R), C=int(t.C), p=float(t.p))
    if fmt == "sell":
        return dict(C=int(t.C), sigma=int(t.sigma))
    if fmt == "csr5":
        return dict(omega=32, sigma=int(t.sigma))
    if fmt == "lav":
        return dict(SIMD_Lanes=int(t.simd_lanes), T=float(t.T), segment_len=int(t.segment_len))
    if fmt == "vhcc":
        return dict(num_threads=int(t.threads))
    return dict(Nthreads=int(t.threads))


def tune(fmt: str, A: F.spMtxCRS, mixed_dtype: torch.dtype | None = None, iters: int = 5):
    """Returns (best parameters, [(parameters, ms), ...]) for format ``fmt``
    built from the CRS matrix ``A``; ``mixed_dtype`` (float32 or bfloat16)
    times the mixed-precision form (on A's values in that type) instead of
    the plain one."""
    if fmt not in _FMT:
        raise ValueError(f"autotune: no candidates for format {fmt!r}")
    mixed = mixed_dtype is not None
    src = A.astype(mixed_dtype) if mixed and A.dtype != mixed_dtype else A
    vt = {torch.float64: _capi.RVVLA_F64, torch.float32: _capi.RVVLA_F32,
          torch.bfloat16: _capi.RVVLA_BF16}[src.dtype]
    lib = _capi.load()
    d = src.desc()
    best, best_ms = _capi.rvvla_tune_params(), C.c_double(0.0)
    cap = 16
    table = (_capi.rvvla_tune_params * cap)()
    table_ms = (C.c_double * cap)()
    ncand = C.c_int(0)
    rc = lib.rvvla_autotune(_FMT[fmt], C.byref(d), vt, 1 if mixed else 0, int(iters), C.byref(best),
                            C.byref(best_ms), table, table_ms, cap, C.byref(ncand), F._stream())
    _capi.check(rc, "rvvla_autotune")
    rows = [(_params(fmt, table[i]), float(table_ms[i])) for i in range(min(ncand.value, cap))]
    return _params(fmt, best), rows
