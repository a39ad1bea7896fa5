"""The device Krylov drivers that restate Krylov.jl's cg and gmres (the
solvers the reference reaches through LinearSolve.jl: test/test_preconditioners.jl
:65,93, README.md:29) against the oracle's restatement (oracle/hs_oracle.c:
hso_cg_kjl, hso_gmres_kjl).  Bar: iteration counts within +-1.

* the reference's own integration cases (test/test_preconditioners.jl:366-560):
  anisotropic convection-diffusion (n = 60^2, eps 0.1) with GMRES, anisotropic
  2D Poisson (n = 100^2, eps 0.1, isSymA) with GMRES for forward/backward and
  CG for symmetric sweeps, partsize 10, packed and view caches, b = ones,
  LinearSolve's default tolerances, through solve(LinearProblem(A, b), alg;
  Pl = P); the reference's assertions (A u ~ b at rtol 0.1, preconditioned
  iterations <= unpreconditioned) plus the +-1 bar against the oracle;
* the 2048-point 1D Laplacian (partsize 16, symmetric packed, CG);
* the 128^3 Poisson operator (CG, partsize 16) and the 96^3 upwind
  convection-diffusion operator (GMRES(30), forward sweep) at full size.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import workloads as W
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

SWEEPS = {"forward": hsb200.ForwardSweep(), "backward": hsb200.BackwardSweep(), "symmetric": hsb200.SymmetricSweep()}
CACHES = {"packed": hsb200.PackedBufferCache(), "view": hsb200.MatrixViewCache()}
TOL = hsb200.DEFAULT_TOL


def builder():
    return hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)


def oracle_iters(kind, A, b, P, memory=None):
    if kind == "cg":
        _, it, _, _ = O.cg_krylovjl(A, b, P, atol=TOL, rtol=TOL)
    else:
        _, it, _, _ = O.gmres_krylovjl(A, b, P, memory=memory or min(A.shape[0], 1024), atol=TOL, rtol=TOL)
    return it


CASES = [("convdiff", "forward", "packed", "gmres"), ("convdiff", "forward", "view", "gmres"),
         ("convdiff", "backward", "packed", "gmres"), ("convdiff", "backward", "view", "gmres"),
         ("poisson2d", "forward", "packed", "gmres"), ("poisson2d", "forward", "view", "gmres"),
         ("poisson2d", "backward", "packed", "gmres"), ("poisson2d", "backward", "view", "gmres"),
         ("poisson2d", "symmetric", "packed", "cg"), ("poisson2d", "symmetric", "view", "cg")]


@pytest.mark.parametrize("mat,sweep,cache,solver", CASES)
def test_reference_integration_cases(mat, sweep, cache, solver):
    if mat == "convdiff":
        A, isSym = W.convection_diffusion_matrix(60, eps=0.1), False
    else:
        A, isSym = W.poisson2d_matrix(100, eps=0.1), True
    b = np.ones(A.shape[0])
    alg = hsb200.KrylovJL_CG() if solver == "cg" else hsb200.KrylovJL_GMRES()
    prob = hsb200.LinearProblem(A, b)
    unprec = hsb200.solve(prob, alg)
    assert np.allclose(A @ unprec.u, b, rtol=1e-1, atol=1e-1)
    P = builder()(A, 10, isSymA=isSym, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], order="reference")
    sol = hsb200.solve(prob, alg, Pl=P)
    assert sol.converged
    assert np.allclose(A @ sol.u, b, rtol=1e-1, atol=1e-1)
    assert sol.iters <= unprec.iters
    ref = O.OracleL1GS(A, 10, isSymA=isSym, sweep=sweep, cache=cache)
    assert abs(sol.iters - oracle_iters(solver, A, b, ref)) <= 1
    assert abs(unprec.iters - oracle_iters(solver, A, b, None)) <= 1


def test_laplacian1d_cg():
    """The 2048-point 1D Laplacian, b = ones, L1GS symmetric packed partsize
    16: Krylov.jl's CG to rtol 1e-8."""
    A = W.poisson_test_matrix(2048)
    b = np.ones(2048)
    P = builder()(A, 16, isSymA=True)
    M = hsb200.DeviceSparseMatrix(A)
    x = torch.zeros(2048, dtype=torch.float64, device="cuda")
    info = hsb200.cg_krylovjl(M, torch.from_numpy(b).cuda(), x, P, rtol=1e-8)
    xo, it, _, rn = O.cg_krylovjl(A, b, O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed"),
                                  rtol=1e-8)
    assert info.converged and abs(info.iterations - it) <= 1
    np.testing.assert_allclose(x.cpu().numpy(), xo, rtol=1e-10, atol=1e-10 * np.abs(xo).max())


def test_gmres_restart_and_memory():
    """Restarted runs (memory 5 and 30) and the itmax cap."""
    A = W.convection_diffusion_matrix(40, eps=0.1)
    b = np.ones(A.shape[0])
    P = builder()(A, 10, sweep=hsb200.ForwardSweep(), order="reference")
    ref = O.OracleL1GS(A, 10, sweep="forward", cache="packed")
    M = hsb200.DeviceSparseMatrix(A)
    bd = torch.from_numpy(b).cuda()
    for memory in (5, 30):
        x = torch.zeros_like(bd)
        info = hsb200.gmres_krylovjl(M, bd, x, P, memory=memory, rtol=1e-8)
        _, it, _, _ = O.gmres_krylovjl(A, b, ref, memory=memory, rtol=1e-8)
        assert info.converged and abs(info.iterations - it) <= 1
    x = torch.zeros_like(bd)
    info = hsb200.gmres_krylovjl(M, bd, x, P, memory=5, rtol=1e-14, itmax=7)
    assert not info.converged and info.iterations == 7


def test_poisson128_cg_full_size():
    A = W.poisson3d_7pt(128)
    b = W.rhs_uniform(A.shape[0])
    P = builder()(A, 16, isSymA=True)
    M = hsb200.DeviceSparseMatrix(A)
    bd = torch.from_numpy(b).cuda()
    x = torch.zeros_like(bd)
    info = hsb200.cg_krylovjl(M, bd, x, P, rtol=1e-8)
    _, it, _, _ = O.cg_krylovjl(A, b, O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed"), rtol=1e-8)
    assert info.converged and abs(info.iterations - it) <= 1


def test_convdiff96_gmres30_full_size():
    A = W.convdiff3d_upwind(96)
    b = W.rhs_uniform(A.shape[0])
    P = builder()(A, 16, sweep=hsb200.ForwardSweep())
    M = hsb200.DeviceSparseMatrix(A)
    bd = torch.from_numpy(b).cuda()
    x = torch.zeros_like(bd)
    info = hsb200.gmres_krylovjl(M, bd, x, P, memory=30, rtol=1e-8)
    _, it, _, _ = O.gmres_krylovjl(A, b, O.OracleL1GS(A, 16, sweep="forward", cache="packed"), memory=30, rtol=1e-8)
    assert info.converged and abs(info.iterations - it) <= 1
