"""GPU: the row-sharded SpMV's default local product (the CRS kernels) in a
one-rank NCCL group (this pool runs one GPU per job; the multi-rank exchange
is covered by the gloo tests on the CPU)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys, socket, datetime
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np, torch, torch.distributed as dist
import oracle as O
from rvvlasparse_b200 import workloads as W
from rvvlasparse_b200.distributed import RowShardedCRS
s = socket.socket(); s.bind(("127.0.0.1", 0)); port = s.getsockname()[1]; s.close()
torch.cuda.set_device(0)
dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{{port}}", rank=0, world_size=1,
                        timeout=datetime.timedelta(seconds=60))
try:
    m, n, Rst, Col, Val = W.powerlaw(200000, seed=8)
    x, y0 = W.vector(n, 1), W.vector(m, 2)
    S = RowShardedCRS(m, n, Rst, Col, Val, device="cuda")
    y = S.spmv(torch.as_tensor(x).cuda(), 0.5, -1.0, torch.as_tensor(y0).cuda())
    torch.cuda.synchronize()
    ref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.5, x, -1.0, y0)
    print(O.normwise_relerr(y.cpu().numpy(), ref))
finally:
    dist.destroy_process_group()
'''


def test_row_sharded_local_product_on_gpu():
    code = CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"))
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-3000:]
    assert float(res.stdout.strip().splitlines()[-1]) < 1e-12
