"""Seeded synthetic workloads (host side; generated by the library's C code).

Shapes follow the measured configurations:

* ``laplace2d(256)``      5-point 2-D Laplacian, n = 65,536, nnz = 326,656;
* ``powerlaw(4194304)``   lognormal rows (mean 16, sigma 1.2, cap 4096), 70 %
  of entries within +-1024 of the diagonal, 30 % uniform, values U[-1,1];
* ``stencil27(128)``      27-point periodic stencil, n = 2,097,152,
  nnz = 56,623,104, values 1 + 0.1 N(0,1);
* ``random_rows``         geometric / Poisson row lengths, uniform columns
  (differentiation and batched workloads).

All return ``(m, n, Rst, Col, Val)`` as numpy arrays (int32, int32, float64).
"""
from __future__ import annotations

import numpy as np

from ._capi import load


def _two_pass(fn, m, *args):
    nz = int(fn(*args, None, None, None))
    if nz < 0:
        raise ValueError("generator rejected its arguments")
    Rst = np.empty(m + 1, dtype=np.int32)
    Col = np.empty(nz, dtype=np.int32)
    Val = np.empty(nz, dtype=np.float64)
    fn(*args, Rst.ctypes.data, Col.ctypes.data, Val.ctypes.data)
    return Rst, Col, Val


def laplace2d(g: int):
    lib = load()
    Rst, Col, Val = _two_pass(lib.rvvla_gen_laplace2d, g * g, g)
    return g * g, g * g, Rst, Col, Val


def stencil27(g: int, seed: int = 3):
    lib = load()
    Rst, Col, Val = _two_pass(lib.rvvla_gen_stencil27, g ** 3, g, seed)
    return g ** 3, g ** 3, Rst, Col, Val


def powerlaw(n: int, mean: float = 16.0, sigma: float = 1.2, cap: int = 4096, band: int = 1024,
             band_frac: float = 0.7, seed: int = 1):
    lib = load()
    Rst, Col, Val = _two_pass(lib.rvvla_gen_powerlaw, n, n, mean, sigma, cap, band, band_frac, seed)
    return n, n, Rst, Col, Val


def random_rows(m: int, n: int, dist: str = "geometric", param: float = 1.0 / 19.0, values: str = "normal",
                seed: int = 5):
    lib = load()
    d = 0 if dist == "geometric" else 1
    v = 0 if values == "normal" else 1
    Rst, Col, Val = _two_pass(lib.rvvla_gen_random_rows, m, m, n, d, param, v, seed)
    return m, n, Rst, Col, Val


def vector(n: int, seed: int = 0, normal: bool = False, lo: float = -1.0, hi: float = 1.0) -> np.ndarray:
    lib = load()
    out = np.empty(n, dtype=np.float64)
    lib.rvvla_gen_vector(n, seed, 1 if normal else 0, lo, hi, out.ctypes.data)
    return out


def batch(count: int = 1024, n_lo: int = 1024, n_hi: int = 65536, avg_lo: float = 4.0, avg_hi: float = 64.0,
          seed: int = 7):
    """The batched workload: ``count`` square matrices, n log-uniform in
    [n_lo, n_hi], average nonzeros per row uniform in [avg_lo, avg_hi], Poisson
    row lengths, uniform random columns, values uniform in [-1, 1]."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), count)).astype(np.int64)
    avgs = rng.uniform(avg_lo, avg_hi, count)
    return [random_rows(int(n), int(n), "poisson", float(a), "uniform", seed=seed * 100003 + i)
            for i, (n, a) in enumerate(zip(ns, avgs))]
