"""GPU parity of the kernels behind the tuning knobs, which are read once
per process: the CRS warp-stream kernel (RVVLA_CRS_KERNEL=stream) and the
CSR5 staging modes (RVVLA_CSR5_STAGING=tma / pipe).  Each runs in a child
process with the knob set and checks fp64, fp32 and mixed products against
the long-double oracle."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r'''
import sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
import numpy as np, torch
import oracle as O, rvvlasparse_b200 as R
from rvvlasparse_b200 import workloads as W
NT = R.SPARSE_OPERATION_NON_TRANSPOSE
fmt = {fmt!r}
worst = {{}}
for empty in (False, True):
    m, n, Rst, Col, Val = W.powerlaw(1 << 17, seed=7)
    if empty:  # drop every 5th row's nonzeros
        ln = np.diff(Rst).astype(np.int64)
        keep = np.repeat(np.arange(m) % 5 != 0, ln)
        ln[np.arange(m) % 5 == 0] = 0
        Rst = np.concatenate([[0], np.cumsum(ln)]).astype(np.int32)
        Col, Val = Col[keep], Val[keep]
    x, y0 = W.vector(n, 3), W.vector(m, 4)
    yref = O.crs_spmv_ld(O.crs(m, n, Rst, Col, Val), 0.5, x, -1.25, y0)
    A64 = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    A32 = A64.astype(torch.float32)
    cases = []
    if fmt == "crs":
        cases = [("f64", A64, False), ("f32", A32, False), ("mixed", A32, True)]
    else:
        for sg in (16, 24):
            for tag, src, mixed in (("f64", A64, False), ("f32", A32, False), ("mixed", A32, True)):
                M = R.spMtxCSR5(); R.convert(M, src, R.convertParams(omega=32, sigma=sg))
                cases.append((f"{{tag}}_s{{sg}}", M, mixed))
    for tag, M, mixed in cases:
        dt = torch.float64 if tag.startswith("f64") else torch.float32
        y = torch.as_tensor(y0).to(dt).cuda()
        fn = R.sparse_mv_mixed if mixed else R.sparse_mv
        st = fn(NT, 0.5, M, R.sparse_matrix_descr(), torch.as_tensor(x).to(dt).cuda(), -1.25, y)
        assert st.code == 0, R.load().rvvla_last_error()
        torch.cuda.synchronize()
        e = O.normwise_relerr(y.cpu().numpy().astype(np.float64), yref)
        worst[tag] = max(worst.get(tag, 0.0), e)
print(repr(worst))
'''


@pytest.mark.parametrize("fmt,knob,value", [("crs", "RVVLA_CRS_KERNEL", "stream"),
                                            ("csr5", "RVVLA_CSR5_STAGING", "tma"),
                                            ("csr5", "RVVLA_CSR5_STAGING", "pipe")])
def test_knob_kernels_match_oracle(fmt, knob, value):
    code = CHILD.format(root=ROOT, tests=os.path.join(ROOT, "tests"), fmt=fmt)
    env = dict(os.environ, **{knob: value})
    res = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=900)
    assert res.returncode == 0, res.stderr[-3000:]
    worst = eval(res.stdout.strip().splitlines()[-1])
    for tag, e in worst.items():
        tol = 1e-12 if tag.startswith("f64") else (1e-6 if tag.startswith("mixed") else 1e-5)
        assert e < tol, (tag, e)
