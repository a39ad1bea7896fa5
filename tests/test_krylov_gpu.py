"""Device PCG / GMRES(30) against the oracle's restatements: iteration counts
agree within +-1 and both reach relative residual 1e-8 (the solution-quality
bar of the reference's LinearSolve tests, tightened)."""
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
    _, it_ref, _ = O.pcg(A, b, O.OracleL1GS(A, ps, isSymA=True, sweep="symmetric", cache=cache), rtol=1e-8)
    assert info.converged
    assert abs(info.iterations - it_ref) <= 1
    assert info.relres <= 1.5e-8
    _, it0, _ = O.pcg(A, b, None)
    assert info.iterations <= it0


def test_pcg_unpreconditioned_and_cheb():
    A = W.poisson3d_7pt(24)
    b = W.rhs_uniform(A.shape[0])
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(A.shape[0], dtype=torch.float64, device="cuda")
    info = hsb200.pcg(M, dev(b), x, None)
    _, it_ref, _ = O.pcg(A, b, None)
    assert info.converged and abs(info.iterations - it_ref) <= 1
    for kind, cfgc in ((4, hsb200.ChebyshevFourth), (1, hsb200.ChebyshevFirst)):
        S = hsb200.build_smoother(cfgc(degree=4), A)
        info = hsb200.pcg(M, dev(b), x, S)
        _, it_ref, _ = O.pcg(A, b, O.OracleChebyshev(A, kind=kind, degree=4, rho=S.rho))
        assert info.converged and abs(info.iterations - it_ref) <= 1 and info.relres <= 1.5e-8


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
    _, it_ref, _ = O.pcg(A, b, ref)
    assert info.converged and abs(info.iterations - it_ref) <= 1 and info.relres <= 1.5e-8


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
    _, it_ref, _ = O.gmres(A, b, O.OracleL1GS(A, 10, sweep="forward", cache=cache), m=30, rtol=1e-8)
    assert info.converged and info.relres <= 1e-8 * 1.01
    assert abs(info.iterations - it_ref) <= 1
    xr = x.cpu().numpy()
    assert np.linalg.norm(b - A @ xr) / np.linalg.norm(b) <= 1.01e-8
