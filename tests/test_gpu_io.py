"""GPU: every built format survives save_format / load_format (arrays equal,
same SpMV result), including a bf16-valued mixed-precision copy."""
import pytest
import torch

import rvvlasparse_b200 as R
from rvvlasparse_b200 import io as RIO
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu
NT = R.SPARSE_OPERATION_NON_TRANSPOSE

BUILDS = [("crs", None, {}), ("hcsr", R.spMtxHCSR, dict(R=500, C=700)), ("sell", R.spMtxSELL_C_Sigma, dict(C=32, sigma=64)),
          ("csr5", R.spMtxCSR5, dict(omega=32, sigma=16)), ("lav", R.spMtxLAV, dict(SIMD_Lanes=8, T=0.2, segment_len=3000)),
          ("vnec", R.spMtxVNEC, dict(threads=16, variant=2)), ("vhcc", R.spMtxVHCC, {}), ("cvr", R.spMtxCVR, {})]


def _arrays(obj):
    return {k: v for k, v in vars(obj).items() if isinstance(v, torch.Tensor)}


@pytest.mark.parametrize("name,cls,params", BUILDS, ids=[b[0] for b in BUILDS])
def test_save_load_format_round_trip(tmp_path, name, cls, params):
    m, n, Rst, Col, Val = W.powerlaw(20000, seed=5)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    M = A if cls is None else cls()
    if cls is not None:
        R.convert(M, A, R.convertParams(**params))
    p = tmp_path / f"{name}.fmt"
    RIO.save_format(M, p)
    M2 = RIO.load_format(p)
    assert type(M2) is type(M)
    a1, a2 = _arrays(M), _arrays(M2)
    assert a1.keys() == a2.keys()
    for k in a1:
        assert a2[k].is_cuda and a1[k].dtype == a2[k].dtype and torch.equal(a1[k], a2[k]), k
    x = torch.as_tensor(W.vector(n, 1)).cuda()
    y1 = torch.as_tensor(W.vector(m, 2)).cuda()
    y2 = y1.clone()
    for mat, y in ((M, y1), (M2, y2)):
        st = R.sparse_mv(NT, 0.5, mat, R.sparse_matrix_descr(), x, 1.5, y)
        assert st.code == 0, R.load().rvvla_last_error()
    torch.cuda.synchronize()
    assert torch.equal(y1, y2) or name == "hcsr"  # HCSR's shared-memory atomics may reorder last bits
    assert torch.allclose(y1, y2, rtol=1e-12, atol=1e-12)


def test_save_load_mixed_bf16(tmp_path):
    m, n, Rst, Col, Val = W.powerlaw(20000, seed=6)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float32)
    M = R.spMtxCSR5()
    R.convert(M, A, R.convertParams(omega=32, sigma=16))
    Mb = M.astype(torch.bfloat16)
    p = tmp_path / "b.fmt"
    RIO.save_format(Mb, p)
    Mb2 = RIO.load_format(p)
    assert Mb2.csr_value.dtype == torch.bfloat16 and torch.equal(Mb.csr_value, Mb2.csr_value)
    x = torch.as_tensor(W.vector(n, 3)).float().cuda()
    y1 = torch.zeros(m, device="cuda")
    y2 = torch.zeros(m, device="cuda")
    for mat, y in ((Mb, y1), (Mb2, y2)):
        assert R.sparse_mv_mixed(NT, 1.0, mat, R.sparse_matrix_descr(), x, 0.0, y).code == 0
    torch.cuda.synchronize()
    assert torch.equal(y1, y2)


def test_load_format_rejects_other_files(tmp_path):
    p = tmp_path / "x.pt"
    torch.save({"hello": 1}, p)
    with pytest.raises(ValueError):
        RIO.load_format(p)
