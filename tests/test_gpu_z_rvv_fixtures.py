"""GPU: the CSR5, VHCC and VNEC products against the outputs of the
reference's own RVV kernels stored in the golden fixtures
(tests/golden/make_golden.py, rvv_outputs: the reference's src/rvv/ sources
built on the oracle's intrinsic stand-in), at the plain tolerances (1e-12
fp64, 1e-5 fp32 normwise)."""
import numpy as np
import pytest
import torch

import rvvlasparse_b200 as R
from helpers import golden_files, golden_id, load_golden, tol_for

pytestmark = pytest.mark.gpu
GOLD = golden_files()
NT = R.SPARSE_OPERATION_NON_TRANSPOSE
TDT = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def run(mat, g):
    y = dev(g["y0"])
    st = R.sparse_mv(NT, g["alpha"], mat, R.sparse_matrix_descr(), dev(g["x"]), g["beta"], y)
    assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    return y.cpu().numpy()


def rel(y, yref):
    den = np.linalg.norm(yref)
    return float(np.linalg.norm(y - yref) / (den if den > 0 else 1.0))


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


def crs(g):
    return R.spMtxCRS.from_host(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], dtype=TDT[g["Val"].dtype])


def test_csr5_matches_reference_rvv_kernel(g):
    C5 = R.spMtxCSR5()
    R.convert(C5, crs(g), R.convertParams(omega=32, sigma=int(g["csr5_sigma"])))
    assert rel(run(C5, g), g["csr5_y"]) < tol_for(g["Val"].dtype)


def test_vhcc_matches_reference_rvv_kernel(g):
    V = R.spMtxVHCC()
    R.convert(V, crs(g), R.convertParams())
    assert rel(run(V, g), g["vhcc_y"]) < tol_for(g["Val"].dtype)


@pytest.mark.parametrize("variant", [0, 1, 2])
def test_vnec_matches_reference_rvv_kernels(g, variant):
    V = R.spMtxVNEC()
    R.convert(V, crs(g), R.convertParams(threads=1, variant=variant))
    assert rel(run(V, g), g[f"vnec{variant}_y"]) < tol_for(g["Val"].dtype)
