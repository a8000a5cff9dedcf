"""GPU parity: CVR builder (SIMD_LEN 32, bit-exact with the oracle builder;
the reference scalar kernel runs on the same layout) and CVR SpMV."""
import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from helpers import golden_files, golden_id, load_golden, tol_for
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
GOLD = golden_files()
NT = R.SPARSE_OPERATION_NON_TRANSPOSE
TDT = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def build(m, n, Rst, Col, Val, threads=0):
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=TDT[np.asarray(Val).dtype])
    V = R.spMtxCVR()
    R.convert(V, A, R.convertParams(Nthreads=threads))
    return V


def run(mat, alpha, x, beta, y0):
    y = dev(y0)
    st = R.sparse_mv(NT, alpha, mat, R.sparse_matrix_descr(), dev(x), beta, y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


@pytest.mark.parametrize("threads", [1, 3, 50])
def test_cvr_builder_and_spmv(g, threads):
    V = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], threads)
    A = O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"])
    o = O.build_cvr(A, 32, threads)
    h = V.to_host()
    assert h["nItems"] == int(o["nItems"])
    assert np.array_equal(h["vPack_vec_cols"].view(np.uint32), o["vPack_vec_cols"])
    assert np.array_equal(h["vPack_vec_vals"], o["vPack_vec_vals"])
    assert np.array_equal(h["vPack_vec_record"], o["vPack_vec_record"])
    assert np.array_equal(h["writeback_pos_record"], o["writeback_pos_record"])
    y = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
    tol = tol_for(g["Val"].dtype)
    yref = O.crs_spmv_ld(A, g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol
    if O.ref_available():  # the reference scalar kernel on the GPU-built layout
        assert O.normwise_relerr(y, O.ref_cvr(o).spmv(g["alpha"], g["x"], g["beta"], g["y0"])) < tol


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_cvr_full_size(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    V = build(m, n, Rst, Col, Val)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(V, 1.0, x, 0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)
