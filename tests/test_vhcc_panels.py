"""Multi-panel VHCC on the CPU: the column split (``column_panels``, run on
CPU tensors), the product it implies composed from the oracle's single-panel
VHCC builder and kernel (src/rvv/spmv_vhcc.cpp:27-397 restated) against the
long-double CSR oracle, and the saved-format round trip of a panel list."""
import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from helpers import golden_files, golden_id, load_golden, tol_for
from rvvlasparse_b200 import formats as F
from rvvlasparse_b200 import io as RIO
from rvvlasparse_b200 import workloads as W

GOLD = golden_files()


def cpu_crs(m, n, Rst, Col, Val):
    return R.spMtxCRS(m, n, len(Col), torch.as_tensor(np.asarray(Rst, np.int32)),
                      torch.as_tensor(np.asarray(Col, np.int32)), torch.as_tensor(np.ascontiguousarray(Val)))


def check_split(m, n, Rst, Col, Val, P):
    parts = F.column_panels(cpu_crs(m, n, Rst, Col, Val), P)
    assert len(parts) == P
    assert parts[0][0] == 0 and parts[-1][1] == n
    for (a0, a1, _), (b0, _, _) in zip(parts, parts[1:]):
        assert a1 == b0 and a0 <= a1
    nz = len(Col)
    assert sum(p.nz for _, _, p in parts) == nz
    colcount = np.bincount(np.asarray(Col, np.int64), minlength=n) if nz else np.zeros(max(n, 1), np.int64)
    for c0, c1, p in parts:
        c = p.Col.numpy()
        assert ((c >= c0) & (c < c1)).all()
        assert p.m == m and p.n == n and p.Rst.numel() == m + 1 and int(p.Rst[-1]) == p.nz
        assert p.nz <= -(-nz // P) + int(colcount.max())  # whole columns: at most one column over the share
    # panels in order, row by row, give back the matrix
    Rst = np.asarray(Rst)
    for i in range(m):
        row_c = np.concatenate([p.Col.numpy()[int(p.Rst[i]):int(p.Rst[i + 1])] for _, _, p in parts])
        row_v = np.concatenate([p.Val.numpy()[int(p.Rst[i]):int(p.Rst[i + 1])] for _, _, p in parts])
        assert np.array_equal(row_c, np.asarray(Col)[Rst[i]:Rst[i + 1]])
        assert np.array_equal(row_v, np.asarray(Val)[Rst[i]:Rst[i + 1]])
    return parts


def composed_spmv(parts, alpha, x, beta, y0, threads):
    """The multi-panel product as sparse_mv runs it: panel after panel, beta
    on the first non-empty panel and 1 after, each through the oracle's
    single-panel VHCC."""
    y = np.array(y0, copy=True)
    first = True
    for _, _, p in parts:
        if p.nz == 0:
            continue
        o = O.build_vhcc(O.crs(p.m, p.n, p.Rst.numpy(), p.Col.numpy(), p.Val.numpy()), threads, 32)
        y = O.spmv(o, alpha, x, beta if first else 1.0, y)
        first = False
    if first:
        y = beta * y
    return y


@pytest.fixture(params=GOLD, ids=[golden_id(p) for p in GOLD])
def g(request):
    return load_golden(request.param)


@pytest.mark.parametrize("P", [1, 2, 3, 7])
def test_column_panels_golden(g, P):
    parts = check_split(g["m"], g["n"], g["Rst"], g["Col"], g["Val"], P)
    y = composed_spmv(parts, g["alpha"], g["x"], g["beta"], g["y0"], 7)
    yref = O.crs_spmv_ld(O.crs(g["m"], g["n"], g["Rst"], g["Col"], g["Val"]), g["alpha"], g["x"], g["beta"], g["y0"])
    assert O.normwise_relerr(y, yref) < tol_for(g["Val"].dtype)


def test_column_panels_balance_powerlaw():
    m, n, Rst, Col, Val = W.powerlaw(1 << 12, seed=5)
    parts = check_split(m, n, Rst, Col, Val, 4)
    sizes = [p.nz for _, _, p in parts]
    assert max(sizes) - min(sizes) <= 2 * int(np.bincount(Col, minlength=n).max())
    x, y0 = W.vector(n, 0), W.vector(m, 1)
    y = composed_spmv(parts, 1.5, x, 0.5, y0, 16)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 1.5, x, 0.5, y0)
    assert O.normwise_relerr(y, yref) < 1e-12


def test_column_panels_more_panels_than_columns():
    Rst = np.array([0, 2, 3, 3, 5], np.int32)
    Col = np.array([0, 2, 1, 0, 2], np.int32)
    Val = np.array([1.0, 2.0, 3.0, 4.0, 5.0])
    parts = check_split(4, 3, Rst, Col, Val, 9)
    assert sum(1 for _, _, p in parts if p.nz) <= 3
    x, y0 = np.array([1.0, -2.0, 0.5]), np.array([1.0, 1.0, 1.0, 1.0])
    y = composed_spmv(parts, 2.0, x, -1.0, y0, 1)
    assert np.allclose(y, 2.0 * np.array([1 + 1.0, -6.0, 0.0, 4 + 2.5]) - 1.0, rtol=0, atol=1e-15)


def test_column_panels_empty_matrix():
    parts = check_split(3, 5, np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0), 4)
    assert all(p.nz == 0 for _, _, p in parts)
    y = composed_spmv(parts, 1.0, np.ones(5), 0.25, np.full(3, 4.0), 1)
    assert np.array_equal(y, np.full(3, 1.0))


def test_column_panels_rejects_zero():
    with pytest.raises(ValueError):
        F.column_panels(cpu_crs(1, 1, [0, 1], [0], [1.0]), 0)


def test_multi_panel_save_load_roundtrip(tmp_path):
    def panel(k):
        p = R.spMtxVHCC()
        p.num_rows, p.num_cols, p.num_entries, p.num_panels = 4, 6, 3 + k, 1
        p.thr_info = torch.arange(10, dtype=torch.int32) + k
        p.vals_arr = torch.linspace(0, 1, 32 + k, dtype=torch.float64)
        return p

    V = R.spMtxVHCC()
    V.num_rows, V.num_cols, V.num_entries, V.num_panels = 4, 6, 7, 2
    V.panels = [panel(0), panel(1)]
    f = tmp_path / "v.fmt"
    RIO.save_format(V, f)
    W2 = RIO.load_format(f, device="cpu")
    assert isinstance(W2, R.spMtxVHCC) and len(W2.panels) == 2
    assert W2.num_panels == 2 and W2.num_entries == 7
    for a, b in zip(V.panels, W2.panels):
        assert torch.equal(a.thr_info, b.thr_info) and torch.equal(a.vals_arr, b.vals_arr)
        assert a.num_entries == b.num_entries
    assert W2.dtype == torch.float64
    assert W2.astype(torch.float32).panels[1].vals_arr.dtype == torch.float32
    with pytest.raises(ValueError):
        W2.desc()
    h = W2.to_host()
    assert len(h["panels"]) == 2 and h["num_panels"] == 2


def test_convert_rejects_zero_panels():
    with pytest.raises(ValueError):
        R.convert(R.spMtxVHCC(), cpu_crs(1, 1, [0, 1], [0], [1.0]), R.convertParams(num_panels=0))
