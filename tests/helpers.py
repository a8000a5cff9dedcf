"""Shared helpers for the tests (golden fixtures, GPU matrices)."""
import glob
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(path):
    d = dict(np.load(path))
    for k in ("m", "n"):
        d[k] = int(d[k])
    for k in ("alpha", "beta"):
        d[k] = float(d[k])
    return d


def golden_id(path):
    return os.path.basename(path)[:-4]


def tol_for(dtype):
    return 1e-12 if np.dtype(dtype) == np.float64 else 1e-5
