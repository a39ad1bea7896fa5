"""The L1GS preconditioner as an AMG smoother (ext/HybridSmoothersAMGExt.jl).

HybridSmoother's smooth! runs two Richardson sweeps residual = A x - b,
correction = P \\ residual, x -= correction (:26-33).  The device version
(one fused residual kernel per sweep plus the L1GS apply) must equal the
oracle restatement bitwise, for the setup the extension uses (SymmetricSweep,
isSymA = false: the DiagonalIndices path of a CSC matrix), for other sweep
counts, and for a non-symmetric matrix; Chebyshev configs smooth through
smooth! itself (:35-49)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import amg
from hsb200 import workloads as W
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu


def _builder():
    return hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)


@pytest.mark.parametrize("mat", ["poisson2d", "convdiff", "variable3d"])
@pytest.mark.parametrize("sweeps", [1, 2, 3])
def test_richardson_smoother_bitwise(mat, sweeps):
    if mat == "poisson2d":
        A = W.poisson2d_matrix(70, eps=0.1)
    elif mat == "convdiff":
        A = W.convection_diffusion_matrix(40, eps=0.1)
    else:
        A = W.variable_diffusion((18, 17, 16), np.random.default_rng(3))
    n = A.shape[0]
    rng = np.random.default_rng(sweeps)
    x0, b = rng.uniform(-1, 1, n), rng.uniform(-1, 1, n)
    S = amg.setup_smoother(_builder(), A, partsize=16)
    x = torch.from_numpy(x0.copy()).cuda()
    amg.smooth_(x, S, torch.from_numpy(b).cuda(), sweeps=sweeps)
    ref = O.amg_richardson(A, O.OracleL1GS(A, 16, isSymA=False, sweep="symmetric", cache="packed"), x0, b, sweeps)
    np.testing.assert_array_equal(x.cpu().numpy(), ref)


def test_richardson_reduces_error_and_repeats():
    """Two calls in a row (the smoother keeps no state between calls) and the
    smoothing property: the error of a Poisson solve goes down."""
    A = W.poisson3d_7pt(20)
    n = A.shape[0]
    xs = np.random.default_rng(0).uniform(-1, 1, n)
    b = A @ xs
    S = amg.setup_smoother(_builder(), A, partsize=8)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    bd = torch.from_numpy(b).cuda()
    P = O.OracleL1GS(A, 8, isSymA=False, sweep="symmetric", cache="packed")
    ref = np.zeros(n)
    errs = [np.linalg.norm(xs)]
    for _ in range(2):
        amg.smooth_(x, S, bd)
        ref = O.amg_richardson(A, P, ref, b)
        np.testing.assert_array_equal(x.cpu().numpy(), ref)
        errs.append(np.linalg.norm(x.cpu().numpy() - xs))
    assert errs[2] < errs[1] < errs[0]


def test_chebyshev_configs_smooth_through_smooth():
    A = W.poisson3d_7pt(12)
    n = A.shape[0]
    b = np.random.default_rng(1).uniform(-1, 1, n)
    for cfg in (hsb200.ChebyshevFourth(degree=3), hsb200.ChebyshevFirst(degree=3)):
        S = amg.setup_smoother(cfg, A)
        x = torch.zeros(n, dtype=torch.float64, device="cuda")
        amg.smooth_(x, S, torch.from_numpy(b).cuda())
        ref = O.OracleChebyshev(A, kind=cfg.kind, degree=3, rho=S.rho).smooth(np.zeros(n), b)
        np.testing.assert_array_equal(x.cpu().numpy(), ref)
