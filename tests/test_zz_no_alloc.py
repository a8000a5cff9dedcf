"""GPU: the allocation-free fp64 CSR5 entry point (static calibrator
scratch) against the ordinary one, called through the C ABI.  Collected
last so that it also runs after every other GPU test in the session."""
import ctypes as C

import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from rvvlasparse_b200 import _capi
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-12  # normwise, fp64


def _matrix(kind):
    if kind == "powerlaw":
        return W.powerlaw(1 << 18, seed=5)
    return W.random_rows(40000, 30000, "poisson", 3.0, seed=9)  # ~5 % empty rows


def _csr5(m, n, Rst, Col, Val):
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    C5 = R.spMtxCSR5()
    R.convert(C5, A, R.convertParams(omega=32, sigma=16))
    return C5


@pytest.mark.parametrize("kind", ["powerlaw", "empty_rows"])
def test_noalloc_matches_ordinary_entry(kind):
    m, n, Rst, Col, Val = _matrix(kind)
    C5 = _csr5(m, n, Rst, Col, Val)
    lib = R.load()
    d = C5.desc()
    x = torch.as_tensor(W.vector(n, 3)).cuda()
    y0 = torch.as_tensor(W.vector(m, 4)).cuda()
    st = torch.cuda.current_stream().cuda_stream
    y_ref = y0.clone()
    assert lib.rvvla_csr5_spmv_f64(C.byref(d), 1.25, x.data_ptr(), -0.5, y_ref.data_ptr(), st) == 0
    outs = []
    for _ in range(2):  # two calls in a row reuse the static scratch
        y = y0.clone()
        rc = lib.rvvla_csr5_spmv_f64_noalloc(C.byref(d), 1.25, x.data_ptr(), -0.5, y.data_ptr(), st)
        assert rc == 0, lib.rvvla_last_error()
        outs.append(y)
    torch.cuda.synchronize()
    ref = y_ref.cpu().numpy()
    for y in outs:
        assert O.normwise_relerr(y.cpu().numpy(), ref) < TOL
    yo = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.25, W.vector(n, 3), -0.5, W.vector(m, 4))
    assert O.normwise_relerr(outs[1].cpu().numpy(), yo) < TOL


def _default_pool():
    from cuda.bindings import runtime as rt

    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess, err
    return rt, pool


def _u64(v):
    from cuda.bindings import driver

    return driver.cuuint64_t(v)


def _pool_attr(rt, pool, attr):
    err, v = rt.cudaMemPoolGetAttribute(pool, attr)
    assert err == rt.cudaError_t.cudaSuccess, err
    return int(v)


def test_noalloc_leaves_the_device_pool_untouched():
    """The defining property: the call takes nothing from the device's
    stream-ordered pool (the ordinary entry's calibrator comes from there).
    The pool's high-water mark is reset before each call and read after it;
    the ordinary entry, measured the same way, shows that the mark sees a
    calibrator allocation.  (The entry's size limit cannot be reached on a
    B200: a launch has at most 48 warps x 148 SMs = 7104 calibrator slots, the
    static array holds 8192.)"""
    m, n, Rst, Col, Val = _matrix("powerlaw")
    C5 = _csr5(m, n, Rst, Col, Val)
    lib = R.load()
    d = C5.desc()
    x = torch.as_tensor(W.vector(n, 3)).cuda()
    y = torch.as_tensor(W.vector(m, 4)).cuda()
    st = torch.cuda.current_stream().cuda_stream
    rt, pool = _default_pool()
    used, high = rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh
    assert lib.rvvla_csr5_spmv_f64_noalloc(C.byref(d), 1.0, x.data_ptr(), 0.0, y.data_ptr(), st) == 0
    torch.cuda.synchronize()
    marks = {}
    for name in ("noalloc", "ordinary"):
        base = _pool_attr(rt, pool, used)
        assert rt.cudaMemPoolSetAttribute(pool, high, _u64(0))[0] == rt.cudaError_t.cudaSuccess
        fn = lib.rvvla_csr5_spmv_f64_noalloc if name == "noalloc" else lib.rvvla_csr5_spmv_f64
        assert fn(C.byref(d), 1.0, x.data_ptr(), 0.0, y.data_ptr(), st) == 0, lib.rvvla_last_error()
        torch.cuda.synchronize()
        marks[name] = (_pool_attr(rt, pool, high), base)
    assert marks["noalloc"][0] == marks["noalloc"][1], marks
    assert marks["ordinary"][0] > marks["ordinary"][1], marks


def test_noalloc_rejects_null_descriptor():
    lib = R.load()
    assert lib.rvvla_csr5_spmv_f64_noalloc(None, 1.0, None, 0.0, None, None) == _capi.RVVLA_ERR_INVALID_ARG
