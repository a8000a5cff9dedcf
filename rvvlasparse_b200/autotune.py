"""Measuring autotuner for the single-matrix formats (no reference counterpart).

``tune(fmt, A, ...)`` builds the format for every candidate parameter set on
the GPU, times ``sparse_mv`` with CUDA events (one warm-up, best of
``iters``) and returns the fastest parameters with the table of all timings.
Candidates:

* ``csr5``  sigma in {8, 16, 24, 32} (omega is fixed to a warp, 32);
* ``sell``  C = 32 (a warp per slice) with sigma in {32, 256, 1024, 8192};
* ``hcsr``  square blocks R = C in {512, 1024, 2000, 4000, 8192}, p = 2;
* ``vhcc``  threads in {nnz/4096, nnz/2048, nnz/1024} (vectors of 32);
* ``cvr``   ranges of {8192, 32768, 131072} nonzeros;
* ``lav``   segment_len in {40000, n/4, n} (SIMD_Lanes 8, T 0.2).

The batched form has its own tuner in the library (``rvvla_batched_autotune``).
"""
from __future__ import annotations

import torch

from . import formats as F

CANDIDATES = {
    "csr5": [dict(omega=32, sigma=s) for s in (8, 16, 24, 32)],
    "sell": [dict(C=32, sigma=s) for s in (32, 256, 1024, 8192)],
    "hcsr": [dict(R=b, C=b, p=2.0) for b in (512, 1024, 2000, 4000, 8192)],
}

_CLASS = {"csr5": F.spMtxCSR5, "sell": F.spMtxSELL_C_Sigma, "hcsr": F.spMtxHCSR, "vhcc": F.spMtxVHCC,
          "cvr": F.spMtxCVR, "lav": F.spMtxLAV}


def _candidates(fmt: str, A: F.spMtxCRS) -> list[dict]:
    if fmt in CANDIDATES:
        return CANDIDATES[fmt]
    if fmt == "vhcc":
        return [dict(num_threads=max(1, A.nz // d)) for d in (4096, 2048, 1024)]
    if fmt == "cvr":
        return [dict(Nthreads=max(1, A.nz // d)) for d in (8192, 32768, 131072)]
    if fmt == "lav":
        return [dict(SIMD_Lanes=8, T=0.2, segment_len=sl) for sl in sorted({40000, max(1, A.n // 4), max(1, A.n)})]
    raise ValueError(f"autotune: no candidates for format {fmt!r}")


def _time(mat, x, y, mixed: bool, iters: int) -> float:
    fn = F.sparse_mv_mixed if mixed else F.sparse_mv
    st = torch.cuda.current_stream()

    def go():
        s = fn(F.SPARSE_OPERATION_NON_TRANSPOSE, 1.0, mat, F.sparse_matrix_descr(), x, 0.0, y)
        if s.code:
            raise RuntimeError(f"autotune: sparse_mv returned {s.code}")

    go()
    best = float("inf")
    for _ in range(iters):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        go()
        e1.record(st)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def tune(fmt: str, A: F.spMtxCRS, mixed_dtype: torch.dtype | None = None, iters: int = 5):
    """Returns (best parameters, [(parameters, ms), ...]) for format ``fmt``
    built from the CRS matrix ``A``; ``mixed_dtype`` (float32 or bfloat16)
    times the mixed-precision form instead of the plain one."""
    cls = _CLASS[fmt]
    mixed = mixed_dtype is not None
    vt = torch.float32 if mixed else A.dtype
    x = torch.empty(A.n, dtype=vt, device=A.Rst.device).uniform_(-1, 1)
    y = torch.empty(A.m, dtype=vt, device=A.Rst.device)
    src = A.astype(torch.float32) if mixed and A.dtype != torch.float32 else A
    table = []
    for params in _candidates(fmt, A):
        M = cls()
        F.convert(M, src, F.convertParams(**params))
        if mixed and mixed_dtype != torch.float32:
            M = M.astype(mixed_dtype)
        table.append((params, _time(M, x, y, mixed, iters)))
        del M
    best = min(table, key=lambda t: t[1])[0]
    return best, table
