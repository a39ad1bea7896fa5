"""Device PCG / GMRES(30) against the oracle's restatements.

Both sides use compensated (Dot2) dot products, separately rounded vector
updates and the same convergence formulas, and the SpMV and preconditioners
are bitwise equal, so the device reproduces the oracle's iterates: iteration
counts are asserted equal (the bar for this path is +-1) and the solutions
equal to 1e-12 relative.  Both reach relative residual 1e-8."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import workloads as W
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


@pytest.mark.parametrize("cache", ["packed", "view"])
@pytest.mark.parametrize("ps", [10, 16])
def test_pcg_l1gs_symmetric(cache, ps):
    A = W.poisson2d_matrix(100, eps=0.1)
    b = np.ones(A.shape[0])
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
        A, ps, isSymA=True, sweep=hsb200.SymmetricSweep(),
        cache_strategy=hsb200.PackedBufferCache() if cache == "packed" else hsb200.MatrixViewCache())
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    info = hsb200.pcg(M, dev(b), x, P, rtol=1e-8)
    x_ref, it_ref, _ = O.pcg(A, b, O.OracleL1GS(A, ps, isSymA=True, sweep="symmetric", cache=cache), rtol=1e-8)
    assert info.converged
    assert info.iterations == it_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-12, atol=0)
    assert info.relres <= 1.5e-8
    _, it0, _ = O.pcg(A, b, None)
    assert info.iterations <= it0


def test_pcg_unpreconditioned_and_cheb():
    A = W.poisson3d_7pt(24)
    b = W.rhs_uniform(A.shape[0])
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    info = hsb200.pcg(M, dev(b), x, None)
    x_ref, it_ref, _ = O.pcg(A, b, None)
    assert info.converged and info.iterations == it_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-12, atol=0)
    for kind, cfgc in ((4, hsb200.ChebyshevFourth), (1, hsb200.ChebyshevFirst)):
        S = hsb200.build_smoother(cfgc(degree=4), A)
        info = hsb200.pcg(M, dev(b), x, S)
        x_ref, it_ref, _ = O.pcg(A, b, O.OracleChebyshev(A, kind=kind, degree=4, rho=S.rho))
        assert info.converged and info.iterations == it_ref and info.relres <= 1.5e-8
        np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-12, atol=0)


def test_pcg_fp32_smoother():
    A = W.poisson3d_7pt(24)
    b = W.rhs_uniform(A.shape[0])
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(A, 16, isSymA=True,
                                                                            precision=np.float32)
    info = hsb200.pcg(M, dev(b), x, P)
    ref = O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed", dtype=np.float32)
    ref.D = O.OracleL1GS(A, 16, isSymA=True).D.astype(np.float32)
    x_ref, it_ref, _ = O.pcg(A, b, ref)
    assert info.converged and info.iterations == it_ref and info.relres <= 1.5e-8
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-12, atol=0)


@pytest.mark.parametrize("cache", ["packed", "view"])
def test_gmres_convection_diffusion(cache):
    A = W.convection_diffusion_matrix(60, eps=0.1)
    b = np.ones(A.shape[0])
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
        A, 10, sweep=hsb200.ForwardSweep(),
        cache_strategy=hsb200.PackedBufferCache() if cache == "packed" else hsb200.MatrixViewCache())
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    info = hsb200.gmres(M, dev(b), x, P, restart=30, rtol=1e-8)
    x_ref, it_ref, _ = O.gmres(A, b, O.OracleL1GS(A, 10, sweep="forward", cache=cache), m=30, rtol=1e-8)
    assert info.converged and info.relres <= 1e-8 * 1.01
    assert info.iterations == it_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-12, atol=0)
    xr = x.cpu().numpy()
    assert np.linalg.norm(b - A @ xr) / np.linalg.norm(b) <= 1.01e-8


def test_pcg_1d_laplacian_workload():
    """The 2048-point 1D Laplacian with L1GS symmetric packed partsize 16 (the
    small workload): ~500 iterations, the longest trajectory in the suite."""
    A = W.poisson_test_matrix(2048)
    b = np.ones(2048)
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(A, 16, isSymA=True)
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(2048, dtype=torch.float64, device="cuda")
    info = hsb200.pcg(M, dev(b), x, P)
    x_ref, it_ref, _ = O.pcg(A, b, O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed"))
    assert info.iterations == it_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=1e-12, atol=0)
