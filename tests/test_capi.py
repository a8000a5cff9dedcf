"""CPU: the C-ABI library loads, exports what include/rvvla.h declares,
validates arguments before touching the GPU, and the workload generators are
deterministic with the documented shapes."""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

from rvvlasparse_b200 import _capi
from rvvlasparse_b200 import workloads as W


def test_library_exports_every_declared_symbol():
    lib = _capi.load()
    declared = _capi.declared_symbols()
    assert len(declared) >= 15
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing


def test_status_strings_and_version():
    lib = _capi.load()
    assert b"sm_100a" in lib.rvvla_version()
    for s in range(9):
        assert lib.rvvla_status_string(s)


def test_null_descriptor_is_rejected_without_gpu():
    lib = _capi.load()
    assert lib.rvvla_crs_spmv_f64(None, 1.0, None, 0.0, None, None) == _capi.RVVLA_ERR_INVALID_ARG
    assert b"null" in lib.rvvla_last_error()
    d = _capi.rvvla_crs(-1, 5, 0, None, None, None, None, 0)
    assert lib.rvvla_crs_spmv_f32(C.byref(d), 1.0, None, 0.0, None, None) == _capi.RVVLA_ERR_INVALID_ARG
    h = _capi.rvvla_hcsr(0, 10, 10, 10, 0, 1, 1, None, None, None, None, None, 0)
    assert lib.rvvla_hcsr_spmv_f64(C.byref(h), 1.0, None, 0.0, None, None) == _capi.RVVLA_ERR_INVALID_ARG
    o = _capi.rvvla_hcsr_owned()
    d = _capi.rvvla_crs(4, 4, 0, None, None, None, None, 0)
    assert lib.rvvla_hcsr_build(C.byref(d), 8, 0, 4, 2.0, C.byref(o), None) == _capi.RVVLA_ERR_INVALID_ARG
    assert b"positive" in lib.rvvla_last_error()


def test_laplace_shape():
    m, n, R, Cc, V = W.laplace2d(256)
    assert m == 65536 and len(Cc) == 326656
    assert R[-1] == 326656 and V.max() == 4.0 and V.min() == -1.0


def test_stencil_shape_and_values():
    m, n, R, Cc, V = W.stencil27(8, seed=3)
    assert m == 512 and len(Cc) == 27 * 512
    assert np.all(np.diff(R) == 27)
    assert abs(V.mean() - 1.0) < 0.02 and 0.08 < V.std() < 0.12
    for i in range(0, m, 37):
        assert np.all(np.diff(Cc[R[i]:R[i + 1]]) > 0)


def test_powerlaw_statistics():
    m, n, R, Cc, V = W.powerlaw(1 << 16, seed=1)
    ln = np.diff(R)
    assert ln.min() >= 1 and ln.max() <= 4096
    assert 14.5 < ln.mean() < 17.5
    rows = np.repeat(np.arange(m), ln)
    assert 0.66 < np.mean(np.abs(Cc - rows) <= 1024) < 0.74
    assert -1 <= V.min() and V.max() <= 1
    for i in range(0, m, 101):
        assert np.all(np.diff(Cc[R[i]:R[i + 1]]) > 0)


def test_generators_deterministic_and_thread_independent():
    a = W.powerlaw(20000, seed=9)
    b = W.powerlaw(20000, seed=9)
    for u, v in zip(a[2:], b[2:]):
        assert np.array_equal(u, v)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    code = ("import sys; sys.path.insert(0, " + repr(root) + "); from rvvlasparse_b200 import workloads as W; "
            "import numpy as np; m,n,R,C,V = W.powerlaw(20000, seed=9); "
            "print(int(R.astype(np.int64).sum()), int(C.astype(np.int64).sum()), repr(float(V.sum())))")
    outs = []
    for nt in ("1", "4"):
        env = dict(os.environ, OMP_NUM_THREADS=nt)
        outs.append(subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                                   check=True).stdout)
    assert outs[0] == outs[1]


def test_random_rows_geometric_mean():
    m, n, R, Cc, V = W.random_rows(100000, 100000, "geometric", 1 / 19, "normal", seed=4)
    ln = np.diff(R)
    assert ln.min() >= 1 and 18.0 < ln.mean() < 20.0


def test_autotune_and_host_copies_validate_before_the_gpu():
    """rvvla_autotune and the staged host copies reject bad arguments
    without touching a device."""
    lib = _capi.load()
    best = _capi.rvvla_tune_params()
    E = _capi.RVVLA_ERR_INVALID_ARG
    assert lib.rvvla_autotune(_capi.RVVLA_FMT_HCSR, None, 0, 0, 1, C.byref(best), None, None, None, 0, None,
                              None) == E
    d = _capi.rvvla_crs(4, 4, 4, None, None, None, None, 0)
    # the mixed form needs F32 or BF16 values, and exists for HCSR / SELL / CSR5 only
    assert lib.rvvla_autotune(_capi.RVVLA_FMT_HCSR, C.byref(d), _capi.RVVLA_F64, 1, 1, C.byref(best), None, None,
                              None, 0, None, None) == E
    assert lib.rvvla_autotune(_capi.RVVLA_FMT_CVR, C.byref(d), _capi.RVVLA_F32, 1, 1, C.byref(best), None, None,
                              None, 0, None, None) == E
    assert lib.rvvla_autotune(99, C.byref(d), _capi.RVVLA_F64, 0, 1, C.byref(best), None, None, None, 0, None,
                              None) == E
    assert lib.rvvla_autotune(_capi.RVVLA_FMT_CSR5, C.byref(d), 7, 0, 1, C.byref(best), None, None, None, 0, None,
                              None) == E
    assert lib.rvvla_copy_h2d(None, None, 16, None) == E
    assert lib.rvvla_copy_d2h(None, None, 16, None) == E
    assert lib.rvvla_copy_h2d(None, None, 0, None) == _capi.RVVLA_OK
