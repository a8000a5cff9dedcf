"""GPU parity: VNEC structures (identical to the oracle's restatement of
include/VNEC.h for the same thread count and variant) and the S / D / L
kernels against the long-double CSR oracle and the restated reference
kernels."""
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
NAMES = {0: "D", 1: "S", 2: "L"}


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def build(m, n, Rst, Col, Val, threads=0, variant=-1):
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=TDT[np.asarray(Val).dtype])
    V = R.spMtxVNEC()
    R.convert(V, A, R.convertParams(threads=threads, variant=variant))
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


@pytest.mark.parametrize("threads", [8, 37])
@pytest.mark.parametrize("variant", [0, 1, 2])
def test_vnec_structure_and_spmv(g, threads, variant):
    V = build(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], threads, variant)
    assert V.vnec_t == variant
    o = O.build_vnec(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), threads, variant)
    h = V.to_host()
    assert np.array_equal(h["thread_coord_start"], o["thread_coord_start"])
    assert np.array_equal(h["thread_coord_end"], o["thread_coord_end"])
    keys = {0: ("ecr_indices", "NEC_NUM", "use_x_ptr", "use_x_indices", "v_row_ptr", "col_start", "val_align"),
            1: ("NEC_NUM", "use_x_ptr", "use_x_indices", "tasks", "task_start", "task_end", "spvv_len",
                "row_begin", "row_end")}.get(variant, ())
    for k in keys:
        assert np.array_equal(h[k], o[k]), k
    if variant == 1:
        assert np.array_equal(h["reorder_col"], o["reorder_col"])
        assert np.array_equal(h["reorder_nnz"], o["reorder_nnz"])
    y = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol_for(g["Val"].dtype)
    assert O.normwise_relerr(y, O.spmv(o, g["alpha"], g["x"], g["beta"], g["y0"])) < tol_for(g["Val"].dtype)
    if variant == 2 and len(g["Col"]) > 0:
        # L runs the CRS lane-run kernel on the analysed plan; without the
        # plan, the merge path over the VNEC threads' coordinates
        assert V.plan is not None and V.plan_kind in (1, 2)
        V.plan, V.plan_kind, V.plan_tiles = None, 0, 0
        y2 = run(V, g["alpha"], g["x"], g["beta"], g["y0"])
        assert O.normwise_relerr(y2, yref) < tol_for(g["Val"].dtype)


def test_vnec_variant_rule_and_ird():
    m, n, Rst, Col, Val = W.powerlaw(60000, seed=3)
    for dt in (np.float64, np.float32):
        V = build(m, n, Rst, Col, Val.astype(dt), 8, -1)
        o = O.build_vnec(O.crs(m, n, Rst, Col, Val.astype(dt)), 8, -1)
        assert V.vnec_t == int(o["vnec_t"])
        assert abs(V.IRD_mat - o["IRD_mat"]) < 1e-6


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_vnec_L_full_size(dt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 22, seed=1)
    Val = Val.astype(dt)
    V = build(m, n, Rst, Col, Val)
    assert V.vnec_t == 2  # m >= 2,000,000 selects L (include/VNEC.h:222-226)
    x, y0 = W.vector(n, 0).astype(dt), W.vector(m, 1).astype(dt)
    y = run(V, 1.0, x, 0.5, y0)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < tol_for(dt)
