"""Parity at the full sizes of the benchmark workloads.

The other GPU tests pin every kernel on small and mid-size matrices; these run
the CUDA path on the workloads' own matrices, where sizes above 2^24 rows or
entries, the SpMV's windows, the number of partition groups per launch and the
ring depths the launchers pick all take their production values:

* 128^3 7-point Poisson (N = 2,097,152): L1GS forward / backward / symmetric,
  packed and view, partsizes 64 and 256, bitwise against the oracle; PCG with
  the partsize-16 symmetric smoother: iteration count and solution against the
  oracle's PCG.
* 96^3 upwind convection-diffusion (non-symmetric CSC, DiagonalIndices path):
  forward sweep, packed and view, bitwise; GMRES(30) iteration count.
* 160^3 27-point lognormal anisotropic diffusion (N = 4,096,000, 109 M
  entries): FP32 smoothers built from the FP64 matrix -- L1GS symmetric packed
  partsize 16 (bitwise against the FP32 oracle with D_Dl1 computed in FP64 and
  rounded) and Chebyshev 1st kind degree 6 (bitwise at the device's rho); the
  FP32-smoother PCG solution against the FP64-smoother one.
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


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def gpu_apply(P, x, dtype=torch.float64):
    xd = dev(x, dtype)
    yd = torch.empty_like(xd)
    hsb200.ldiv_(yd, P, xd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.fixture(scope="module")
def poisson128():
    A = W.poisson3d_7pt(128)
    return A, W.rhs_uniform(A.shape[0])


@pytest.fixture(scope="module")
def convdiff96():
    A = W.convdiff3d_upwind(96)
    return A, W.rhs_uniform(A.shape[0])


@pytest.fixture(scope="module")
def aniso160():
    A = W.aniso27_lognormal(160)
    return A, W.rhs_uniform(A.shape[0])


@pytest.mark.parametrize("ps", [64, 256])
@pytest.mark.parametrize("cache", ["packed", "view"])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_poisson128_l1gs_bitwise(poisson128, ps, cache, sweep):
    A, x = poisson128
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache=cache)
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], order="reference")
    np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))


def test_poisson128_pcg_iterations(poisson128):
    """PCG to 1e-8 with the headline smoother: the device driver's iteration
    count equals the oracle driver's (the bar is +-1) and the solutions agree."""
    A, b = poisson128
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(A, 16, isSymA=True)
    M = hsb200.DeviceSparseMatrix(A)
    bd = dev(b)
    x = torch.zeros_like(bd)
    info = hsb200.pcg(M, bd, x, P, rtol=1e-8)
    x_ref, it_ref, _ = O.pcg(A, b, O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed"))
    assert info.converged and abs(info.iterations - it_ref) <= 1
    assert info.relres <= 1.5e-8   # true residual; the driver stops on the recursive one
    xs = x.cpu().numpy()
    assert np.linalg.norm(xs - x_ref) <= 1e-12 * np.linalg.norm(x_ref)


@pytest.mark.parametrize("cache", ["packed", "view"])
def test_convdiff96_forward_bitwise(convdiff96, cache):
    A, x = convdiff96
    ref = O.OracleL1GS(A, 16, sweep="forward", cache=cache)
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, 16, sweep=hsb200.ForwardSweep(), cache_strategy=CACHES[cache])
    np.testing.assert_array_equal(P.D_DL1, ref.D)
    np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))


def test_convdiff96_gmres_iterations(convdiff96):
    """GMRES(30) to 1e-8 with the forward-sweep packed smoother: iteration
    count within +-1 of the oracle driver's."""
    A, b = convdiff96
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, 16, sweep=hsb200.ForwardSweep(), cache_strategy=hsb200.PackedBufferCache())
    M = hsb200.DeviceSparseMatrix(A)
    bd = dev(b)
    x = torch.zeros_like(bd)
    info = hsb200.gmres(M, bd, x, P, restart=30, rtol=1e-8)
    _, it_ref, _ = O.gmres(A, b, O.OracleL1GS(A, 16, sweep="forward", cache="packed"), m=30)
    assert info.converged and abs(info.iterations - it_ref) <= 1


def test_aniso160_fp32_l1gs_bitwise(aniso160):
    A, x = aniso160
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, 16, isSymA=True, sweep=hsb200.SymmetricSweep(), precision=np.float32)
    D64 = O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed").D
    np.testing.assert_array_equal(P.D_DL1, D64.astype(np.float32))
    ref = O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed", dtype=np.float32)
    ref.D = D64.astype(np.float32)
    want = ref.ldiv(x.astype(np.float32))
    np.testing.assert_array_equal(gpu_apply(P, x.astype(np.float32), torch.float32), want)
    # FP64 vectors in and out of the FP32 smoother (the mixed-precision PCG's call)
    np.testing.assert_array_equal(gpu_apply(P, x, torch.float64), want.astype(np.float64))


def test_aniso160_fp32_cheb1_bitwise(aniso160):
    A, b = aniso160
    S = hsb200.build_smoother(hsb200.ChebyshevFirst(degree=6, precision=np.float32), A)
    ref = O.OracleChebyshev(A, kind=1, degree=6, dtype=np.float32, rho=S.rho)
    n = A.shape[0]
    xd = torch.zeros(n, dtype=torch.float32, device="cuda")
    hsb200.smooth_(xd, S, dev(b, torch.float32))
    np.testing.assert_array_equal(xd.cpu().numpy(), ref.smooth(np.zeros(n, np.float32), b.astype(np.float32)))
    zd = torch.empty(n, dtype=torch.float64, device="cuda")
    hsb200.ldiv_(zd, S, dev(b))
    np.testing.assert_array_equal(zd.cpu().numpy(), ref.apply(b.astype(np.float32)).astype(np.float64))


@pytest.mark.parametrize("smoother", ["l1gs", "cheb1"])
def test_aniso160_fp32_solve_error(aniso160, smoother):
    """FP32 smoother inside FP64 PCG to 1e-8: the solution differs from the
    FP64-smoother solve by at most 1e-6 relative.  Both satisfy
    ||b - A x|| <= 1e-8 ||b||; the bound leaves room for the operator's
    conditioning (the measured difference is about 2e-9 for L1GS and 4e-13 for
    Chebyshev)."""
    A, b = aniso160
    M = hsb200.DeviceSparseMatrix(A)
    bd = dev(b)
    sols = {}
    for prec in (None, np.float32):
        if smoother == "l1gs":
            P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
                A, 16, isSymA=True, precision=prec)
        else:
            P = hsb200.build_smoother(hsb200.ChebyshevFirst(degree=6, precision=prec), A)
        x = torch.zeros_like(bd)
        info = hsb200.pcg(M, bd, x, P, rtol=1e-8)
        assert info.converged and info.relres <= 1.5e-8
        sols[prec] = x.cpu().numpy()
        del P
    err = np.linalg.norm(sols[np.float32] - sols[None]) / np.linalg.norm(sols[None])
    assert err <= 1e-6, err
