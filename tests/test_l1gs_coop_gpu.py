"""GPU parity of the packed sweeps that reorder a row's sum, against the
oracle: the cooperative sweeps (several lanes per partition: the column-block
kernel, csrc/l1gs_coop_kernel.cuh, for 4, 16 and 32 lanes; the blocked
kernel, csrc/l1gs_blk.cu, for 8 lanes and partsizes that are multiples of 8)
and the rows kernel with partial sums (order="any", csrc/l1gs.cu).

Forward sweeps add each row's terms in the reference's ascending order and are
compared bitwise.  Backward and symmetric sweeps add them in descending order,
so they are compared at the contract's tolerance: relative 1e-12 for FP64
(elementwise, with an absolute floor of 1e-12 * max|y|), 1e-5 for FP32.
Packed-buffer introspection returns the reference layout, so SLbuffer/SUbuffer
are compared bitwise like the thread-per-partition kernels'.
"""
import numpy as np
import pytest
import scipy.sparse as sp

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import workloads as W
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

SWEEPS = {"forward": hsb200.ForwardSweep(), "backward": hsb200.BackwardSweep(), "symmetric": hsb200.SymmetricSweep()}


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def gpu_apply(P, x, dtype=torch.float64):
    xd = dev(x, dtype)
    yd = torch.empty_like(xd)
    hsb200.ldiv_(yd, P, xd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def device_error_clear():
    import ctypes
    code = ctypes.c_int32()
    hsb200._lib.check(hsb200.lib().hs_device_error(None, ctypes.byref(code)))
    return code.value


@pytest.fixture(autouse=True)
def _no_device_errors():
    device_error_clear()
    yield
    assert device_error_clear() == 0, "a bounded device wait timed out"


def check(got, want, sweep, rtol):
    if sweep == "forward":
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=rtol, atol=rtol * np.abs(want).max())


def random_matrix(n, density, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=rng, format="csc")
    A.data = rng.uniform(-1, 1, A.nnz)
    A = A + sp.diags(rng.uniform(3, 5, n) + abs(A).sum(axis=1).A.ravel())
    return W._canon(A.tocsc())


# (partsize, lanes per partition, n): ragged last partitions, groups with
# padding partitions, every instantiated (lanes, rows-per-lane) pair -- exact
# fits for 4 lanes, exact and other partsizes for 16 and 32; 8 lanes: the
# blocked kernel at one to 64 row blocks per partition, partsizes that are
# multiples of 8 and padded ones
COOP_CASES = [(16, 4, 1000), (32, 4, 999), (64, 4, 3000), (32, 8, 2048), (64, 8, 3000), (128, 8, 4000),
              (8, 8, 777), (24, 8, 1001), (40, 8, 999), (56, 8, 3001), (256, 8, 5000), (512, 8, 4100),
              (12, 8, 999), (31, 8, 2000), (33, 8, 1500), (100, 8, 2345), (300, 8, 2500),
              (5, 16, 301), (17, 16, 500), (33, 16, 1111), (64, 16, 4000), (100, 16, 2345), (256, 16, 4000),
              (2, 32, 50), (20, 32, 700), (128, 32, 3001), (256, 32, 4000), (300, 32, 2500), (512, 32, 3000)]


@pytest.mark.parametrize("ps,tpp,n", COOP_CASES)
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_coop_random_fp64(ps, tpp, n, sweep):
    A = random_matrix(n, min(0.5, 12.0 / n), ps * 7 + n)
    x = np.random.default_rng(n).uniform(-1, 1, n)
    for fmt, isSym in (("csc", False), ("csr", False), ("csc", True)):
        M = A.asformat(fmt)
        ref = O.OracleL1GS(M, ps, isSymA=isSym, sweep=sweep, cache="packed")
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
            M, ps, isSymA=isSym, sweep=SWEEPS[sweep], threads_per_part=tpp)
        assert P.threads_per_part == tpp
        np.testing.assert_array_equal(P.D_DL1, ref.D)
        check(gpu_apply(P, x), ref.ldiv(x), sweep, 1e-12)
        if sweep != "backward":
            np.testing.assert_array_equal(P.SLbuffer, ref.SL)
        if sweep != "forward":
            np.testing.assert_array_equal(P.SUbuffer, ref.SU)


@pytest.mark.parametrize("ps,tpp", [(16, 4), (33, 16), (64, 16), (130, 32), (32, 8), (72, 8), (256, 8), (31, 8), (100, 8)])
@pytest.mark.parametrize("sweep", ["forward", "symmetric"])
def test_coop_fp32_and_mixed(ps, tpp, sweep):
    A = W.poisson2d_matrix(40, eps=0.3)
    x = np.random.default_rng(ps).uniform(-1, 1, A.shape[0])
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=8)
    A32 = A.astype(np.float32)
    ref = O.OracleL1GS(A32, ps, isSymA=True, sweep=sweep, cache="packed")
    P = b(A32, ps, isSymA=True, sweep=SWEEPS[sweep], threads_per_part=tpp)
    check(gpu_apply(P, x.astype(np.float32), torch.float32), ref.ldiv(x.astype(np.float32)), sweep, 1e-5)
    Pm = b(A, ps, isSymA=True, sweep=SWEEPS[sweep], precision=np.float32, threads_per_part=tpp)
    D64 = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="packed").D
    np.testing.assert_array_equal(Pm.D_DL1, D64.astype(np.float32))
    refm = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="packed", dtype=np.float32)
    refm.D = D64.astype(np.float32)
    want = refm.ldiv(x.astype(np.float32)).astype(np.float64)
    check(gpu_apply(Pm, x, torch.float64), want, sweep, 1e-5)


@pytest.mark.parametrize("tpp", [8, 32])
def test_coop_nonsymmetric_csc(tpp):
    """The DiagonalIndices path feeds the same cooperative streams."""
    A = W.convdiff3d_upwind(20)
    x = W.rhs_uniform(A.shape[0])
    for sweep in ("forward", "backward", "symmetric"):
        ref = O.OracleL1GS(A, 64, sweep=sweep, cache="packed")
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, 64, sweep=SWEEPS[sweep], threads_per_part=tpp)
        check(gpu_apply(P, x), ref.ldiv(x), sweep, 1e-12)


def test_coop_in_place_and_host_apply():
    A = W.poisson3d_7pt(40)
    x = np.random.default_rng(1).uniform(-1, 1, A.shape[0])
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=8)(
        A, 64, isSymA=True, threads_per_part=16)
    want = gpu_apply(P, x)
    xd = dev(x)
    hsb200.ldiv_(xd, P, xd)
    np.testing.assert_array_equal(xd.cpu().numpy(), want)
    got = np.empty_like(x)
    hsb200.ldiv_(got, P, x)   # host vectors: chunks of whole cooperative groups
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("ps,tpp", [(40, 16), (64, 16), (40, 8), (64, 8)])
def test_coop_nonfinite_input(ps, tpp):
    """inf/NaN in x reach the same rows as in the reference (forward: bitwise,
    NaN positions included; backward/symmetric: the same non-finite pattern).
    900 rows: the last partition is short, so padding rows meet the inf."""
    A = W.poisson2d_matrix(30, eps=0.5)
    x = np.random.default_rng(5).uniform(-1, 1, A.shape[0])
    x[ps + 10] = np.inf
    x[3] = np.nan
    x[A.shape[0] - 2] = -np.inf
    for sweep in ("forward", "backward", "symmetric"):
        ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="packed").ldiv(x)
        got = gpu_apply(hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
            A, ps, isSymA=True, sweep=SWEEPS[sweep], threads_per_part=tpp), x)
        np.testing.assert_array_equal(np.isnan(got), np.isnan(ref))
        np.testing.assert_array_equal(np.isinf(got), np.isinf(ref))
        fin = np.isfinite(ref)
        check(got[fin], ref[fin], sweep, 1e-12)


def test_coop_rejects_unsupported():
    A = W.poisson_test_matrix(100)
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=8)
    with pytest.raises(NotImplementedError, match="not provided"):
        b(A, 100, isSymA=True, threads_per_part=4)    # 25 rows per lane: not instantiated
    with pytest.raises(NotImplementedError, match="not provided"):
        b(A, 5, isSymA=True, threads_per_part=8)      # 8 lanes: partsizes from 8 (padded to multiples of 8)
    with pytest.raises(NotImplementedError, match="not provided"):
        b(A, 36, isSymA=True, threads_per_part=4)     # 4 lanes: exact fits only
    with pytest.raises(ValueError, match="threads per partition"):
        b(A, 16, isSymA=True, threads_per_part=3)
    # a view cache always runs one thread per partition
    P = b(A, 16, isSymA=True, cache_strategy=hsb200.MatrixViewCache(), threads_per_part=8)
    assert P.threads_per_part == 1


@pytest.mark.parametrize("ps,tpp", [(64, 8), (64, 16), (256, 32)])
def test_coop_poisson128_full_size(ps, tpp):
    """The 128^3 workload at full size: forward bitwise, symmetric to 1e-12."""
    A = W.poisson3d_7pt(128)
    x = W.rhs_uniform(A.shape[0])
    for sweep in ("forward", "symmetric"):
        ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="packed")
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, ps, isSymA=True, sweep=SWEEPS[sweep], threads_per_part=tpp)
        check(gpu_apply(P, x), ref.ldiv(x), sweep, 1e-12)


ROWS_ANY_CASES = [(32, 2048), (33, 1111), (40, 900), (64, 3000), (100, 2345), (256, 4000), (300, 2500)]


@pytest.mark.parametrize("ps,n", ROWS_ANY_CASES)
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_rows_partial_sums_fp64(ps, n, sweep):
    """Thread per partition with four partial sums per row (order="any")."""
    A = random_matrix(n, min(0.5, 12.0 / n), ps * 11 + n)
    x = np.random.default_rng(n + 1).uniform(-1, 1, n)
    for fmt, isSym in (("csc", False), ("csr", False), ("csc", True)):
        M = A.asformat(fmt)
        ref = O.OracleL1GS(M, ps, isSymA=isSym, sweep=sweep, cache="packed")
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
            M, ps, isSymA=isSym, sweep=SWEEPS[sweep], threads_per_part=1, order="any")
        assert P.order == "any"
        np.testing.assert_allclose(gpu_apply(P, x), ref.ldiv(x), rtol=1e-12,
                                   atol=1e-12 * np.abs(ref.ldiv(x)).max())


@pytest.mark.parametrize("ps", [64, 256])
def test_rows_partial_sums_fp32_and_full_size(ps):
    A = W.poisson3d_7pt(128)
    x = W.rhs_uniform(A.shape[0])
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep="symmetric", cache="packed")
    P = b(A, ps, isSymA=True, threads_per_part=1, order="any")
    want = ref.ldiv(x)
    np.testing.assert_allclose(gpu_apply(P, x), want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    Pm = b(A, ps, isSymA=True, threads_per_part=1, order="any", precision=np.float32)
    refm = O.OracleL1GS(A, ps, isSymA=True, sweep="symmetric", cache="packed", dtype=np.float32)
    refm.D = ref.D.astype(np.float32)
    wm = refm.ldiv(x.astype(np.float32)).astype(np.float64)
    np.testing.assert_allclose(gpu_apply(Pm, x), wm, rtol=1e-5, atol=1e-5 * np.abs(wm).max())


def test_reference_order_is_default_and_bitwise():
    """Without options the library keeps the reference's order (bitwise)."""
    A = W.poisson3d_7pt(30)
    x = W.rhs_uniform(A.shape[0])
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(A, 64, isSymA=True,
                                                                             order="reference")
    assert P.order == "reference" and P.threads_per_part == 1
    ref = O.OracleL1GS(A, 64, isSymA=True, sweep="symmetric", cache="packed")
    np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))
    with pytest.raises(ValueError, match="reference summation order"):
        hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, 64, isSymA=True, order="reference", threads_per_part=8)


@pytest.mark.parametrize("ps", [31, 32, 64, 100, 256])
def test_blocked_forward_keeps_reference_order(ps):
    """The blocked kernel's forward sweep adds every row's terms in the
    reference's order: with order="reference" the library runs it (8 lanes
    per partition) and the result is bitwise; without options a forward
    sweep at these partsizes runs it too and reports the reference order."""
    A = W.poisson3d_7pt(30)
    x = W.rhs_uniform(A.shape[0])
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep="forward", cache="packed").ldiv(x)
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)
    for kw in (dict(order="reference", threads_per_part=8), dict(order="reference"), {}):
        P = b(A, ps, isSymA=True, sweep=hsb200.ForwardSweep(), **kw)
        assert P.threads_per_part == 8 and P.order == "reference", kw
        np.testing.assert_array_equal(gpu_apply(P, x), ref)
