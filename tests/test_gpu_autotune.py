"""GPU: the single-matrix autotuner times every candidate and its choice is
a valid, correct configuration."""
import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from rvvlasparse_b200 import autotune as AT
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("fmt", ["csr5", "sell", "hcsr", "vhcc", "cvr", "lav"])
def test_tune_picks_fastest_valid_candidate(fmt):
    m, n, Rst, Col, Val = W.powerlaw(1 << 16, seed=2)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val)
    best, table = AT.tune(fmt, A, iters=2)
    assert len(table) >= 3 and all(ms > 0 for _, ms in table)
    assert best == min(table, key=lambda t: t[1])[0]
    M = AT._CLASS[fmt]()
    R.convert(M, A, R.convertParams(**best))
    x = W.vector(n, 1)
    y = torch.zeros(m, dtype=torch.float64, device="cuda")
    assert R.sparse_mv(R.SPARSE_OPERATION_NON_TRANSPOSE, 1.0, M, R.sparse_matrix_descr(),
                       torch.as_tensor(x).cuda(), 0.0, y).code == 0
    ref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.0, x, 0.0, np.zeros(m))
    assert O.normwise_relerr(y.cpu().numpy(), ref) < 1e-12


def test_tune_mixed_bf16_csr5():
    m, n, Rst, Col, Val = W.stencil27(32, seed=3)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val)
    best, table = AT.tune("csr5", A, mixed_dtype=torch.bfloat16, iters=2)
    assert best["sigma"] in (8, 16, 24, 32) and len(table) == 4
