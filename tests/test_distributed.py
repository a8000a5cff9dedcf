"""Row-sharded SpMV (one process per GPU) checked on the CPU with gloo ranks:
nonzero-balanced row ranges, the x all-gather over uneven ranges, and the
assembled y against the oracle.  The local products use the oracle's CRS
SpMV here (a CPU stand-in for the GPU kernel the ranks use by default)."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from rvvlasparse_b200.distributed import row_bounds  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q, exchange, overlap, kind):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle as O
    from rvvlasparse_b200 import workloads as W
    from rvvlasparse_b200.distributed import RowShardedCRS

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        m, n, Rst, Col, Val = _matrix(kind)
        x = W.vector(n, 1)
        y0 = W.vector(m, 2)

        def local(which, alpha, xv, beta, y_local):  # the oracle's CRS product on one block of this rank
            R_, C_, V_ = S.diag if which == "diag" else S.off
            A = O.crs(S.local_rows, len(xv), R_, C_, V_)
            y_local.copy_(torch.as_tensor(O.crs_spmv_ld(A, alpha, xv.numpy(), beta, y_local.numpy())))

        S = RowShardedCRS(m, n, Rst, Col, Val, device="cpu", local_spmv=local, exchange=exchange, overlap=overlap)
        xl = torch.as_tensor(x[S.r0:S.r1].copy())
        ghost = S.gather_x(xl)
        if exchange == "halo":  # exactly the remote columns the rows reference
            need = np.unique(S.Col_l[(S.Col_l < S.r0) | (S.Col_l >= S.r1)])
            assert np.array_equal(ghost.numpy(), x[need])
        yl = torch.as_tensor(y0[S.r0:S.r1].copy())
        S.spmv(xl, 0.5, -2.0, yl)
        S.spmv(xl, 1.0, 1.0, yl)  # a second product: same collective order on every rank
        q.put((rank, S.r0, S.r1, yl.numpy(), S.exchanged_per_spmv))
    finally:
        dist.destroy_process_group()


def _matrix(kind):
    from rvvlasparse_b200 import workloads as W

    if kind == "powerlaw":
        return W.powerlaw(6000, seed=4)
    return W.laplace2d(60)  # banded: rank k needs one grid line from each neighbour


def _run(world, exchange, overlap, kind):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q, exchange, overlap, kind)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


@pytest.mark.parametrize("world,exchange,overlap,kind", [(2, "halo", True, "powerlaw"), (3, "halo", False, "powerlaw"),
                                                         (3, "allgather", True, "powerlaw"),
                                                         (2, "allgather", False, "powerlaw"),
                                                         (3, "halo", True, "banded")])
def test_row_sharded_spmv_on_gloo_ranks(world, exchange, overlap, kind):
    """Diagonal block while the exchange is in flight, then the off-diagonal
    block on the ghosts; both exchanges, with and without overlap, against
    the long-double oracle on the whole matrix."""
    import oracle as O
    from rvvlasparse_b200 import workloads as W

    res = _run(world, exchange, overlap, kind)
    m, n, Rst, Col, Val = _matrix(kind)
    A = O.crs(m, n, Rst, Col, Val)
    x, y0 = W.vector(n, 1), W.vector(m, 2)
    y1 = O.crs_spmv_ld(A, 0.5, x, -2.0, y0)
    y2 = O.crs_spmv_ld(A, 1.0, x, 1.0, y1)
    y = np.zeros(m)
    for rank, r0, r1, yl, _ in res:
        y[r0:r1] = yl
    assert res[0][1] == 0 and res[-1][2] == m
    assert O.normwise_relerr(y, y2) < 1e-14
    if kind == "banded":  # the halo of a 5-point stencil: one grid line per neighbour
        assert all(sent <= 2 * 60 for *_, sent in res)


def test_row_bounds_balance_and_edges():
    Rst = np.array([0, 10, 11, 12, 13, 40, 41, 42], dtype=np.int64)  # one long row
    for world in (1, 2, 3, 7, 10):
        b = row_bounds(Rst, world)
        assert len(b) == world + 1 and b[0] == 0 and b[-1] == 7 and np.all(np.diff(b) >= 0)
    from rvvlasparse_b200 import workloads as W
    m, n, R, C, V = W.powerlaw(50000, seed=3)
    b = row_bounds(R, 8)
    share = np.diff(np.asarray(R, np.int64)[b]) / len(C)
    assert np.all(np.abs(share - 1 / 8) < 0.02)
    with pytest.raises(ValueError):
        row_bounds(R, 0)
