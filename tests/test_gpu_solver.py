"""GPU: conjugate gradients over the CRS path (fused SpMV-dot and fused
update-dot) against scipy's direct solution and a numpy CG with the same
recurrences."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla
import torch

import rvvlasparse_b200 as R
from rvvlasparse_b200 import solvers as S
from rvvlasparse_b200 import workloads as W

pytestmark = pytest.mark.gpu


def numpy_cg(A, b, rtol, max_iter):
    x = np.zeros_like(b)
    r = b - A @ x
    p = r.copy()
    rr = r @ r
    bb = b @ b
    it = 0
    while np.sqrt(rr / bb) > rtol and it < max_iter:
        q = A @ p
        alpha = rr / (p @ q)
        x += alpha * p
        r -= alpha * q
        rr_new = r @ r
        p = r + (rr_new / rr) * p
        rr = rr_new
        it += 1
    return x, it


def laplace(g, shift=0.0):
    m, n, Rst, Col, Val = W.laplace2d(g)
    Val = Val.copy()
    if shift:
        for i in range(m):  # diagonal shift keeps A symmetric positive definite
            k = Rst[i] + np.searchsorted(Col[Rst[i]:Rst[i + 1]], i)
            Val[k] += shift
    return m, n, Rst, Col, Val


@pytest.mark.parametrize("g,shift", [(40, 0.0), (128, 0.5)])
def test_cg_fp64_matches_direct_and_numpy_cg(g, shift):
    m, n, Rst, Col, Val = laplace(g, shift)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    As = sp.csr_matrix((Val, Col, Rst), shape=(m, n))
    b = W.vector(n, 7)
    x, it, rel = S.cg(A, torch.as_tensor(b).cuda(), rtol=1e-10, max_iter=5000, check_every=1)
    xh = x.cpu().numpy()
    assert rel <= 1e-10
    assert np.linalg.norm(b - As @ xh) / np.linalg.norm(b) < 1e-9  # true residual
    xd = spla.spsolve(As.tocsc(), b)
    assert np.linalg.norm(xh - xd) / np.linalg.norm(xd) < 1e-7
    _, it_np = numpy_cg(As, b, 1e-10, 5000)
    assert abs(it - it_np) <= 2
    # bitwise reproducible, and check_every only changes where it stops
    x2, it2, _ = S.cg(A, torch.as_tensor(b).cuda(), rtol=1e-10, max_iter=5000, check_every=1)
    assert it2 == it and torch.equal(x, x2)
    x3, it3, rel3 = S.cg(A, torch.as_tensor(b).cuda(), rtol=1e-10, max_iter=5000, check_every=16)
    assert it <= it3 < it + 16 and rel3 <= 1e-10


def test_cg_fp32_and_initial_guess():
    m, n, Rst, Col, Val = laplace(64, 0.25)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val.astype(np.float32), dtype=torch.float32)
    b = W.vector(n, 3).astype(np.float32)
    x, it, rel = S.cg(A, torch.as_tensor(b).cuda(), rtol=1e-5, max_iter=2000, check_every=4)
    As = sp.csr_matrix((Val, Col, Rst), shape=(m, n))
    assert rel <= 1e-5
    assert np.linalg.norm(b - As @ x.double().cpu().numpy()) / np.linalg.norm(b) < 1e-4
    # starting from the solution: no iteration needed
    _, it0, rel0 = S.cg(A, torch.as_tensor(b).cuda(), x0=x, rtol=1e-3, max_iter=10, check_every=1)
    assert it0 == 0 and rel0 <= 1e-3


def test_cg_max_iter_and_errors():
    m, n, Rst, Col, Val = laplace(64)
    A = R.spMtxCRS.from_host(m, n, Rst, Col, Val, dtype=torch.float64)
    b = torch.as_tensor(W.vector(n, 1)).cuda()
    _, it, rel = S.cg(A, b, rtol=1e-14, max_iter=5, check_every=3)
    assert it == 5 and rel > 1e-14
    lib = R.load()
    import ctypes as C
    d = A.desc()  # no plan
    it_, rr_ = C.c_int64(), C.c_double()
    x = torch.zeros_like(b)
    assert lib.rvvla_cg_f64(C.byref(d), b.data_ptr(), x.data_ptr(), 10, 1e-8, 1, C.byref(it_), C.byref(rr_),
                            torch.cuda.current_stream().cuda_stream) != 0
    m2, n2, R2, C2, V2 = W.random_rows(100, 80, "geometric", 0.2, "normal", seed=2)
    A2 = R.spMtxCRS.from_host(m2, n2, R2, C2, V2, dtype=torch.float64)
    with pytest.raises(ValueError):
        S.cg(A2, torch.zeros(m2, dtype=torch.float64, device="cuda"))


@pytest.mark.parametrize("dt", [np.float64, np.float32])
def test_spmv_dot_fused(dt):
    # y = A x and x^T A x in one pass, on matrices with and without empty rows
    for empty in (False, True):
        m, n, Rst, Col, Val = W.powerlaw(1 << 16, seed=9)
        if empty:
            ln = np.diff(Rst).astype(np.int64)
            drop = np.arange(m) % 7 == 0
            keep = np.repeat(~drop, ln)
            ln[drop] = 0
            Rst = np.concatenate([[0], np.cumsum(ln)]).astype(np.int32)
            Col, Val = Col[keep], Val[keep]
        tdt = torch.float64 if dt == np.float64 else torch.float32
        A = R.spMtxCRS.from_host(m, n, Rst, Col, Val.astype(dt), dtype=tdt)
        x = torch.as_tensor(W.vector(n, 4).astype(dt)).cuda()
        y, d = S.spmv_dot(A, x)
        As = sp.csr_matrix((Val.astype(np.float64), Col, Rst), shape=(m, n))
        xh = x.double().cpu().numpy()
        yref = As @ xh
        tol = 1e-12 if dt == np.float64 else 1e-5
        assert np.linalg.norm(y.double().cpu().numpy() - yref) / np.linalg.norm(yref) < tol
        dref = xh @ yref
        assert abs(float(d.item()) - dref) / abs(dref) < (1e-11 if dt == np.float64 else 1e-4)
        y2, d2 = S.spmv_dot(A, x)
        assert torch.equal(y, y2) and torch.equal(d, d2)


# ---------------------------------------------------------------- BiCGStab

def numpy_bicgstab(A, b, rtol, max_iter):
    """Unpreconditioned BiCGStab with the recurrences of rvvla_bicgstab_*."""
    x = np.zeros_like(b)
    r = b - A @ x
    rh = r.copy()
    p = np.zeros_like(b)
    v = np.zeros_like(b)
    rho, alpha, omega, beta = rh @ r, 1.0, 1.0, 0.0
    bb = b @ b
    rr = r @ r
    it = 0
    while np.sqrt(rr / bb) > rtol and it < max_iter:
        p = r + beta * (p - omega * v)
        v = A @ p
        alpha = rho / (rh @ v)
        s = r - alpha * v
        t = A @ s
        omega = (t @ s) / (t @ t)
        x += alpha * p + omega * s
        r = s - omega * t
        rho_new = rh @ r
        beta = (rho_new / rho) * (alpha / omega)
        rho = rho_new
        rr = r @ r
        it += 1
    return x, it


def convection_diffusion(g, c):
    """5-point Laplacian plus a first-order convection term of strength c:
    non-symmetric, diagonally dominant."""
    e = np.ones(g)
    T = sp.diags([-(1 + c) * e[:-1], 4 * e, -(1 - c) * e[:-1]], [-1, 0, 1])
    I = sp.identity(g)
    S1 = sp.diags([-e[:-1], -e[:-1]], [-1, 1])
    A = (sp.kron(I, T) + sp.kron(S1, I)).tocsr()
    A.sort_indices()
    return A


@pytest.mark.parametrize("g,c", [(48, 0.3), (160, 0.7)])
def test_bicgstab_fp64_matches_direct_and_numpy(g, c):
    As = convection_diffusion(g, c)
    m = As.shape[0]
    A = R.spMtxCRS.from_host(m, m, As.indptr.astype(np.int32), As.indices.astype(np.int32), As.data,
                             dtype=torch.float64)
    b = W.vector(m, 11)
    x, it, rel, bd = S.bicgstab(A, torch.as_tensor(b).cuda(), rtol=1e-10, max_iter=5000, check_every=1)
    xh = x.cpu().numpy()
    assert not bd and rel <= 1e-10
    assert np.linalg.norm(b - As @ xh) / np.linalg.norm(b) < 1e-9  # true residual
    xd = spla.spsolve(As.tocsc(), b)
    assert np.linalg.norm(xh - xd) / np.linalg.norm(xd) < 1e-7
    _, it_np = numpy_bicgstab(As, b, 1e-10, 5000)
    assert abs(it - it_np) <= 3
    # bitwise reproducible; a later check only runs a few more iterations
    x2, it2, _, _ = S.bicgstab(A, torch.as_tensor(b).cuda(), rtol=1e-10, max_iter=5000, check_every=1)
    assert it2 == it and torch.equal(x, x2)
    _, it10, rel10, _ = S.bicgstab(A, torch.as_tensor(b).cuda(), rtol=1e-10, max_iter=5000, check_every=10)
    assert it <= it10 < it + 10 and rel10 <= 1e-10


def test_bicgstab_fp32_and_limits():
    As = convection_diffusion(64, 0.5)
    m = As.shape[0]
    Rst, Col = As.indptr.astype(np.int32), As.indices.astype(np.int32)
    A32 = R.spMtxCRS.from_host(m, m, Rst, Col, As.data.astype(np.float32), dtype=torch.float32)
    b = W.vector(m, 12)
    x, it, rel, bd = S.bicgstab(A32, torch.as_tensor(b.astype(np.float32)).cuda(), rtol=1e-5, max_iter=2000)
    assert not bd and rel <= 1e-5
    xh = x.double().cpu().numpy()
    assert np.linalg.norm(b - As @ xh) / np.linalg.norm(b) < 1e-4
    # max_iter stops it; an exact initial guess needs no iteration
    A64 = R.spMtxCRS.from_host(m, m, Rst, Col, As.data, dtype=torch.float64)
    _, it3, rel3, _ = S.bicgstab(A64, torch.as_tensor(b).cuda(), rtol=1e-14, max_iter=3, check_every=2)
    assert it3 == 3 and rel3 > 1e-14
    xd = spla.spsolve(As.tocsc(), b)
    _, it0, rel0, _ = S.bicgstab(A64, torch.as_tensor(b).cuda(), x0=torch.as_tensor(xd).cuda(), rtol=1e-8)
    assert it0 == 0 and rel0 <= 1e-8


def test_bicgstab_rejects_bad_arguments():
    As = convection_diffusion(8, 0.1)
    m = As.shape[0]
    A = R.spMtxCRS.from_host(m, m, As.indptr.astype(np.int32), As.indices.astype(np.int32), As.data,
                             dtype=torch.float64)
    b = torch.ones(m, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        S.bicgstab(A, b[:-1])
    with pytest.raises(ValueError):
        S.bicgstab(A, b, check_every=0)
    Rn = np.array([0, 1, 2], np.int32)
    An = R.spMtxCRS.from_host(2, 3, Rn, np.array([0, 2], np.int32), np.ones(2), dtype=torch.float64)
    with pytest.raises(ValueError):
        S.bicgstab(An, torch.ones(2, dtype=torch.float64, device="cuda"))
