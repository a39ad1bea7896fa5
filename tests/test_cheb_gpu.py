"""GPU parity of mul! (CSR SpMV) and the Chebyshev smoothers against the oracle.

Mirrors test/test_chebyshev.jl (l1 row sums, 0 < rho <= 1, residual decrease,
monotone over applications, degree ordering, a* ordering, 1st vs 4th kind,
repeatability) and adds bitwise parity of the fused step kernels.  rho is a
parallel-sum estimate on the device, so parity of the recurrence is checked at
the device's rho (bitwise) and rho itself against the oracle's power iteration
(relative 1e-12).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import workloads as W
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def csr(A):
    R = A.tocsr()
    R.sort_indices()
    return R


@pytest.mark.parametrize("mat", ["poisson3d", "aniso27", "convdiff", "random"])
def test_spmv_modes_bitwise(mat):
    if mat == "poisson3d":
        A = W.poisson3d_7pt(20)
    elif mat == "aniso27":
        A = W.aniso27_lognormal(14)
    elif mat == "convdiff":
        A = W.convdiff3d_upwind(18)
    else:
        import scipy.sparse as sp
        rng = np.random.default_rng(5)
        A = W._canon(sp.random(3001, 3001, density=0.01, random_state=rng, format="csc") + sp.eye(3001))
    R = csr(A)
    n = A.shape[0]
    x = np.random.default_rng(1).uniform(-1, 1, n)
    y0 = np.random.default_rng(2).uniform(-1, 1, n)
    for dt, tdt in ((np.float64, torch.float64), (np.float32, torch.float32)):
        M = hsb200.DeviceSparseMatrix(A, dtype=dt)
        v = R.data.astype(dt)
        xd = dev(x, tdt)
        yd = torch.empty(n, dtype=tdt, device="cuda")
        hsb200.mul_(yd, M, xd)
        np.testing.assert_array_equal(yd.cpu().numpy(), O.spmv(R.indptr, R.indices, v, x.astype(dt)))
        yd = dev(y0, tdt)
        hsb200.mul_(yd, M, xd, -1.0, 1.0)
        ref = O.spmv_sub(R.indptr, R.indices, v, x.astype(dt), y0.astype(dt).copy())
        np.testing.assert_array_equal(yd.cpu().numpy(), ref)
    # general alpha, beta against numpy
    M = hsb200.DeviceSparseMatrix(A)
    yd = dev(y0)
    hsb200.mul_(yd, M, dev(x), 0.5, -2.0)
    np.testing.assert_allclose(yd.cpu().numpy(), 0.5 * (A @ x) - 2.0 * y0, rtol=1e-12, atol=1e-12)


def build_pair(A, kind, degree, precision=None, eig="power"):
    cfgc = hsb200.ChebyshevFourth if kind == 4 else hsb200.ChebyshevFirst
    S = hsb200.build_smoother(cfgc(degree=degree, eig=eig, precision=precision), A)
    ref = O.OracleChebyshev(A, kind=kind, degree=degree, dtype=precision or np.float64, rho=S.rho)
    return S, ref


def test_rho_and_astar_against_oracle():
    for A in (W.poisson_test_matrix(100), W.poisson3d_7pt(16), W.aniso27_lognormal(12)):
        S = hsb200.build_smoother(hsb200.ChebyshevFourth(degree=4), A)
        ref = O.OracleChebyshev(A, kind=4, degree=4)
        assert abs(S.rho - ref.rho) <= 1e-12 * ref.rho
        assert 0 < S.rho <= 1
    for k in range(1, 9):
        S = hsb200.build_smoother(hsb200.ChebyshevFirst(degree=k), W.poisson_test_matrix(10))
        assert abs(S.a - O.cheb1_astar(k)) <= 1e-15
        assert 0 < S.a < 1


@pytest.mark.parametrize("kind", [4, 1])
@pytest.mark.parametrize("degree", [1, 2, 4, 6, 8])
def test_smooth_bitwise_fp64(kind, degree):
    A = W.poisson3d_7pt(20)
    n = A.shape[0]
    S, ref = build_pair(A, kind, degree)
    b = np.random.default_rng(degree).uniform(-1, 1, n)
    x0 = np.random.default_rng(degree + 10).uniform(-1, 1, n)
    xd, bd = dev(x0), dev(b)
    hsb200.smooth_(xd, S, bd)
    np.testing.assert_array_equal(xd.cpu().numpy(), ref.smooth(x0.copy(), b))
    # apply form z = smooth!(0, S, r) (the PCG adapter)
    zd = torch.empty_like(bd)
    hsb200.ldiv_(zd, S, bd)
    np.testing.assert_array_equal(zd.cpu().numpy(), ref.apply(b))


@pytest.mark.parametrize("kind", [4, 1])
def test_smooth_bitwise_fp32_and_mixed(kind):
    A = W.aniso27_lognormal(16)
    n = A.shape[0]
    S, ref = build_pair(A, kind, 6, precision=np.float32)
    b = np.random.default_rng(3).uniform(-1, 1, n)
    xd = torch.zeros(n, dtype=torch.float32, device="cuda")
    hsb200.smooth_(xd, S, dev(b, torch.float32))
    np.testing.assert_array_equal(xd.cpu().numpy(), ref.smooth(np.zeros(n, np.float32), b.astype(np.float32)))
    zd = torch.empty(n, dtype=torch.float64, device="cuda")
    hsb200.ldiv_(zd, S, dev(b))
    np.testing.assert_array_equal(zd.cpu().numpy(), ref.apply(b.astype(np.float32)).astype(np.float64))


@pytest.mark.parametrize("kind", [4, 1])
def test_residual_properties(kind):
    """test/test_chebyshev.jl:50-95, :115-158 on the GPU."""
    N = 300
    A = W.poisson_test_matrix(N)
    b = np.ones(N)
    res = []
    cfgc = hsb200.ChebyshevFourth if kind == 4 else hsb200.ChebyshevFirst
    for degree in (1, 2, 4, 8):
        S = hsb200.build_smoother(cfgc(degree=degree), A)
        xd = torch.zeros(N, dtype=torch.float64, device="cuda")
        hsb200.smooth_(xd, S, dev(b))
        r = np.linalg.norm(b - A @ xd.cpu().numpy())
        assert r < np.linalg.norm(b)
        res.append(r)
    assert all(res[i] >= res[i + 1] for i in range(3))
    A = W.poisson_test_matrix(200)
    b = np.random.default_rng(42).random(200)
    S = hsb200.build_smoother(cfgc(degree=4), A)
    xd = torch.zeros(200, dtype=torch.float64, device="cuda")
    prev = np.linalg.norm(b)
    for _ in range(10):
        hsb200.smooth_(xd, S, dev(b))
        cur = np.linalg.norm(b - A @ xd.cpu().numpy())
        assert cur < prev
        prev = cur
    assert prev / np.linalg.norm(b) < 0.9


def test_lanczos_bounds():
    A = W.poisson3d_7pt(16)
    S = hsb200.build_smoother(hsb200.ChebyshevFourth(degree=4, eig="lanczos"), A)
    info = S.info
    assert 0 < info.lanczos_min < info.lanczos_max <= 1.0 + 1e-12
    assert info.lanczos_max >= info.rho_power * (1 - 1e-6)
    assert S.rho == info.lanczos_max


def test_power_iteration_large_grid():
    """A matrix with more row blocks than the power iteration has partial
    slots (80^3 rows = 2000 blocks of 256 > 1184): the kernel must stride over
    row blocks and rho must still match the oracle's."""
    A = W.poisson3d_7pt(80)
    S = hsb200.build_smoother(hsb200.ChebyshevFourth(degree=4), A)
    ref = O.OracleChebyshev(A, kind=4, degree=4)
    assert abs(S.rho - ref.rho) <= 1e-12 * ref.rho
    assert 0.5 < S.rho <= 1
