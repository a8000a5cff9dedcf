"""GPU parity of the batched form: many CRS matrices (empty rows, an empty
matrix, uneven sizes) with k right-hand sides in one persistent launch, in
every per-matrix mapping (CSR with 1..32 threads per row, SELL-C-sigma), as
chosen by the autotuner, and replayed from a CUDA graph; each matrix's block
of Y against the long-double oracle, column by column."""
import numpy as np
import pytest
import torch

import oracle as O
import rvvlasparse_b200 as R
from helpers import tol_for
from rvvlasparse_b200 import batched as B
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
TDT = {np.float64: torch.float64, np.float32: torch.float32}


def make_batch(dt, count=24, seed=3):
    host = W.batch(count, 64, 3000, 0.5, 70.0, seed=seed)
    host.append(W.random_rows(0, 10, "poisson", 3.0, "uniform", seed=1))  # an empty matrix
    host.append(W.random_rows(300, 500, "geometric", 1.0 / 200.0, "uniform", seed=2))  # long rows, m != n
    mats = [R.spMtxCRS.from_host(m, n, Rst, Col, Val.astype(dt), dtype=TDT[dt]) for m, n, Rst, Col, Val in host]
    return host, mats


def check(host, batch, X, Y, Y0, alpha, beta, dt):
    k = batch.k
    Xh, Yh = X.cpu().numpy(), Y.cpu().numpy()
    for i, (m, n, Rst, Col, Val) in enumerate(host):
        if m == 0:
            continue
        A = O.crs(m, n, Rst, Col, Val.astype(dt))
        xs = Xh[batch.x_off[i]:batch.x_off[i + 1]].reshape(n, k)
        ys = Yh[batch.y_off[i]:batch.y_off[i + 1]].reshape(m, k)
        y0 = Y0[batch.y_off[i]:batch.y_off[i + 1]].reshape(m, k)
        for r in range(k):
            ref = O.crs_spmv_ld(A, alpha, xs[:, r], beta, y0[:, r])
            assert O.normwise_relerr(ys[:, r], ref) < tol_for(dt), (i, r)


def vectors(batch, dt, seed):
    X = torch.as_tensor(W.vector(batch.x_len, seed).astype(dt)).cuda()
    Y0 = W.vector(batch.y_len, seed + 1).astype(dt)
    return X, Y0


@pytest.mark.parametrize("dt", [np.float64, np.float32])
@pytest.mark.parametrize("k", [1, 4, 8, 32])
@pytest.mark.parametrize("layout", ["csr", "sell", "mixed"])
def test_batched_mappings(dt, k, layout):
    host, mats = make_batch(dt)
    n = len(mats)
    rng = np.random.default_rng(k)
    if layout == "csr":
        mode = np.zeros(n, np.int32)
        param = rng.choice([1, 2, 4, 8, 16, 32], n).astype(np.int32)
    elif layout == "sell":
        mode = np.ones(n, np.int32)
        param = rng.choice([32, 64, 256], n).astype(np.int32)
    else:
        mode = rng.integers(0, 2, n).astype(np.int32)
        param = np.where(mode == 0, 4, 128).astype(np.int32)
    batch = B.SpMVBatch(mats, k=k, mode=mode, param=param)
    X, Y0 = vectors(batch, dt, 5)
    Y = torch.as_tensor(Y0).cuda()
    assert batch.spmv(1.25, X, -0.5, Y) == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    check(host, batch, X, Y, Y0, 1.25, -0.5, dt)


@pytest.mark.parametrize("k", [1, 8])
def test_batched_autotuned_and_graph(k):
    dt = np.float32
    host, mats = make_batch(dt, count=32, seed=9)
    batch = B.SpMVBatch(mats, k=k, tune=True)
    assert batch.tuned_ms is not None and batch.tuned_ms > 0
    assert set(np.unique(batch.mode)) <= {0, 1}
    X, Y0 = vectors(batch, dt, 7)
    Y = torch.empty(batch.y_len, dtype=torch.float32, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        g = batch.graph(2.0, X, 0.0, Y)
        for _ in range(2):
            Y.fill_(float("nan"))  # beta = 0 must not read Y
            g.launch()
    s.synchronize()
    check(host, batch, X, Y, np.zeros(batch.y_len, dt), 2.0, 0.0, dt)
    del g


def test_batched_rejects_bad_k():
    _, mats = make_batch(np.float64, count=2)
    with pytest.raises(ValueError):
        B.SpMVBatch(mats, k=3)
