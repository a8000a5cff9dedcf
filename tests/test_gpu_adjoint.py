"""GPU parity: the adjoint forms — transposed CRS built on the GPU (bit-exact
with the oracle's counting-sort transpose), dx = A^T g (against the fp64
oracle and the reference scalar CRS SpMV run on the transposed matrix),
SDDMM dvalues (bit-exact) and the autograd binding under gradcheck."""
import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from helpers import golden_files, golden_id, load_golden, tol_for
from rvvlasparse_b200 import autograd as AG
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = golden_files()
TDT = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def pattern(m, n, Rst, Col, dt):
    return AG.CrsPattern(m, n, dev(np.asarray(Rst, np.int32)), dev(np.asarray(Col, np.int32)), TDT[np.dtype(dt)])


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def test_transpose_bit_exact(g):
    dt = g["Val"].dtype
    P = pattern(g["m"], g["n"], g["Rst"], g["Col"], dt)
    vals = dev(g["Val"])
    gvec = dev(g["y0"])
    P.adjoint_x_refreshed(vals, gvec, 1.0)  # refreshes A^T's values
    torch.cuda.synchronize()
    t = {k: v.cpu().numpy() for k, v in P.transposed().items()}
    o = O.transpose(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]))
    for k in ("Rst", "Col", "perm", "Val"):
        assert np.array_equal(t[k], o[k]), k


def test_adjoint_x_and_sddmm(g):
    m, n, dt = g["m"], g["n"], g["Val"].dtype
    P = pattern(m, n, g["Rst"], g["Col"], dt)
    vals = dev(g["Val"])
    gv = W.vector(m, 11).astype(dt)
    xv = g["x"].astype(dt)
    dx = P.adjoint_x(vals, dev(gv), 1.5).cpu().numpy()
    A = O.crs(m, n, g["Rst"], g["Col"], g["Val"])
    At = O.transpose(A)
    ref = O.crs_spmv_ld(At, 1.5, gv, 0.0, np.zeros(n))
    assert O.normwise_relerr(dx, ref) < tol_for(dt)
    # through the re-gathered A^T values: the same sums in the same order
    dx2 = P.adjoint_x_refreshed(vals, dev(gv), 1.5).cpu().numpy()
    assert np.array_equal(dx, dx2)
    if O.ref_available():  # the reference's own CRS kernel on A^T
        y = O.ref_crs(At).spmv(1.5, gv, 0.0, np.zeros(n, dt))
        assert O.normwise_relerr(dx, y) < tol_for(dt)
    dv = P.sddmm(dev(gv), dev(xv)).cpu().numpy()
    assert np.array_equal(dv, O.sddmm(A, gv, xv).astype(dt))


def test_gradcheck_fp64():
    # the generator of the adjoint workload at its gradcheck size: n = 2048,
    # geometric row lengths with mean 19 (~40k nonzeros), N(0,1) values
    m, n, Rst, Col, Val = W.random_rows(2048, 2048, "geometric", 1.0 / 19.0, "normal", seed=21)
    assert 30000 < len(Col) < 50000
    P = pattern(m, n, Rst, Col, np.float64)
    v = dev(Val).requires_grad_(True)
    x = dev(W.vector(n, 22)).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda vv, xx: AG.spmv(P, vv, xx, 0.75), (v, x), eps=1e-6, atol=1e-8,
                                    rtol=1e-6, fast_mode=False)


def test_backward_matches_oracle_fp32_large():
    # the adjoint workload: n = 1,048,576, geometric rows (mean 19), uniform
    # random columns, N(0,1) values, fp32; upstream gradient N(0,1)
    m, n, Rst, Col, Val = W.random_rows(1 << 20, 1 << 20, "geometric", 1.0 / 19.0, "normal", seed=31)
    Val = Val.astype(np.float32)
    P = pattern(m, n, Rst, Col, np.float32)
    v = dev(Val).requires_grad_(True)
    xh = W.vector(n, 32, normal=True).astype(np.float32)
    x = dev(xh).requires_grad_(True)
    y = AG.spmv(P, v, x)
    gh = W.vector(m, 33, normal=True).astype(np.float32)
    y.backward(dev(gh))
    A = O.crs(m, n, Rst, Col, Val)
    yo = O.crs_spmv_ld(A, 1.0, xh, 0.0, np.zeros(m))
    assert O.normwise_relerr(y.detach().cpu().numpy(), yo) < 1e-5
    dxo = O.crs_spmv_ld(O.transpose(A), 1.0, gh, 0.0, np.zeros(n))
    assert O.normwise_relerr(x.grad.cpu().numpy(), dxo) < 1e-5
    assert np.array_equal(v.grad.cpu().numpy(), O.sddmm(A, gh, xh).astype(np.float32))


def test_transpose_rejects_bad_value_size():
    import ctypes as C

    from rvvlasparse_b200 import _capi

    lib = R.load()
    d = _capi.rvvla_crs(4, 4, 0, None, None, None, None, 0, 0)
    out = _capi.rvvla_transpose_owned()
    assert lib.rvvla_csr_transpose(C.byref(d), 3, C.byref(out), None) == _capi.RVVLA_ERR_INVALID_ARG


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_sparse_mv_transpose_operation(g, dt):
    """sparse_mv(SPARSE_OPERATION_TRANSPOSE) on a CRS matrix: y = a*A^T b + c*y
    (the reference declares the operation and ignores it)."""
    m, n = g["m"], g["n"]
    Val = g["Val"].astype(dt)
    A = R.spMtxCRS.from_host(m, n, g["Rst"], g["Col"], Val, dtype=TDT[np.dtype(dt)])
    b = W.vector(m, 41).astype(dt)
    y0 = W.vector(n, 42).astype(dt)
    y = dev(y0)
    st = R.sparse_mv(R.SPARSE_OPERATION_TRANSPOSE, 0.5, A, R.sparse_matrix_descr(), dev(b), 2.0, y)
    assert st.code == 0, R.load().rvvla_last_error()
    ref = O.crs_spmv_ld(O.transpose(O.crs(m, n, g["Rst"], g["Col"], Val)), 0.5, b, 2.0, y0)
    assert O.normwise_relerr(y.cpu().numpy(), ref) < tol_for(dt)
    A.Val.mul_(-1.0)  # values changed in place: the cached transpose follows
    y = dev(y0)
    assert R.sparse_mv(R.SPARSE_OPERATION_TRANSPOSE, 0.5, A, R.sparse_matrix_descr(), dev(b), 2.0, y).code == 0
    ref = O.crs_spmv_ld(O.transpose(O.crs(m, n, g["Rst"], g["Col"], -Val)), 0.5, b, 2.0, y0)
    assert O.normwise_relerr(y.cpu().numpy(), ref) < tol_for(dt)
