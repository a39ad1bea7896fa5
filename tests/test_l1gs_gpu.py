"""GPU parity of the L1GS apply (libhsb200, sm_100a) against the CPU oracle.

Mirrors the reference's GPU suite (test/gpu/gpu.jl:111-357: known answers,
blocks x threads invariance, eta, non-symmetric CSC, partsize 3) and adds
bitwise parity on random and stencil matrices.  Bar: bit-exact for FP64 and
FP32 (the kernels keep the reference's per-row ascending order with separately
rounded multiply/add, and so does the oracle).
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import workloads as W
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))
SWEEPS = {"forward": hsb200.ForwardSweep(), "backward": hsb200.BackwardSweep(), "symmetric": hsb200.SymmetricSweep()}
CACHES = {"packed": hsb200.PackedBufferCache(), "view": hsb200.MatrixViewCache()}


def kat(name):
    return np.array(KATS[name]["value"])


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


SWEEP_KAT = {"forward": "gpu_y_exp_fwd", "backward": "gpu_y_exp_bwd", "symmetric": "gpu_y_exp_sym"}


@pytest.mark.parametrize("fmt", ["csc", "csr"])
@pytest.mark.parametrize("cache", ["packed", "view"])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_algorithm_kat(fmt, cache, sweep):
    """test_sym_result (test/gpu/gpu.jl:21-61, :113-357): D_DL1, packed buffers
    and P \\ x for blocks x threads layouts."""
    A = W.poisson_test_matrix(9).asformat(fmt)
    x = np.arange(9, dtype=np.float64)
    for blocks in (1, 2, 5, 10):
        for threads in (1, 3, 10):
            b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=threads, blocks=blocks)
            P = b(A, 2, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache])
            np.testing.assert_array_equal(P.D_DL1, kat("D_Dl1_exp"))
            if cache == "packed":
                if sweep != "backward":
                    np.testing.assert_array_equal(P.SLbuffer, kat("SLbuffer_exp"))
                if sweep != "forward":
                    np.testing.assert_array_equal(P.SUbuffer, kat("SUbuffer_exp"))
            np.testing.assert_array_equal(gpu_apply(P, x), kat(SWEEP_KAT[sweep]))
            # P \ x on host vectors: the generic ldiv! path with copies
            np.testing.assert_array_equal(hsb200.backslash(P, x), kat(SWEEP_KAT[sweep]))


def test_symmetric_type_input():
    A = W.poisson_test_matrix(9)
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=4, blocks=2)
    P = b(hsb200.Symmetric(sp.triu(A).tocsc(), "U"), 2, sweep=hsb200.SymmetricSweep())
    np.testing.assert_array_equal(gpu_apply(P, np.arange(9.0)), kat("gpu_y_exp_sym"))


def test_eta_parameter():
    A = W.poisson_test_matrix(9)
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=2, blocks=2)
    for eta, key in ((2.0, "D_Dl1_exp"), (3.0, "D_Dl1_eta3"), (1.0, "D_Dl1_exp")):
        P = b(A, 2, eta=eta, sweep=hsb200.ForwardSweep(), cache_strategy=hsb200.PackedBufferCache())
        np.testing.assert_array_equal(P.D_DL1, kat(key))
        np.testing.assert_array_equal(P.SLbuffer, kat("SLbuffer_exp"))
    P = b(A, 2, eta=2.0, sweep=hsb200.ForwardSweep(), cache_strategy=hsb200.PackedBufferCache())
    np.testing.assert_array_equal(gpu_apply(P, np.arange(9.0)), kat("y_exp_fwd"))


@pytest.mark.parametrize("cache", ["packed", "view"])
def test_nonsymmetric_csc(cache):
    A2 = W.poisson_test_matrix(9).tolil()
    A2[0, 7] = -1.0
    A2[1, 7] = -1.0
    A2 = W._canon(A2.tocsc())
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=2, blocks=2)
    x = np.arange(9.0)
    P = b(A2, 2, sweep=hsb200.ForwardSweep(), cache_strategy=CACHES[cache])
    np.testing.assert_array_equal(P.D_DL1, kat("D_Dl1_exp2"))
    if cache == "packed":
        np.testing.assert_array_equal(P.SLbuffer, kat("SLbuffer_exp"))
    np.testing.assert_allclose(gpu_apply(P, x), kat("y2_fwd_exp"), rtol=0, atol=1e-15)
    np.testing.assert_array_equal(P.diag_indices, O.diag_indices(A2.indptr, A2.indices, A2.data))
    P = b(A2, 2, sweep=hsb200.BackwardSweep(), cache_strategy=CACHES[cache])
    np.testing.assert_array_equal(P.D_DL1, kat("D_Dl1_exp2"))
    if cache == "packed":
        np.testing.assert_array_equal(P.SUbuffer, kat("SUbuffer_exp"))
    np.testing.assert_allclose(gpu_apply(P, x), kat("y2_bwd_exp"), rtol=0, atol=1e-15)


def test_partsize3_layout():
    A = W.poisson_test_matrix(9)
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=2, blocks=2)(
        A, 3, sweep=hsb200.ForwardSweep(), cache_strategy=hsb200.PackedBufferCache())
    np.testing.assert_array_equal(P.D_DL1, kat("D_Dl1_exp"))
    np.testing.assert_array_equal(P.SLbuffer, kat("SLbuffer_exp_ps3"))


def test_singular_diagonal():
    A = W.poisson_test_matrix(6).tolil()
    A[3, 3] = 0.0
    A = A.tocsc()
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=2, blocks=2)
    with pytest.raises(hsb200.SingularException) as e:
        b(A, 2, sweep=hsb200.ForwardSweep())
    assert e.value.col == 4


def test_bad_arguments():
    A = W.poisson_test_matrix(9)
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=2, blocks=2)
    with pytest.raises(ValueError, match="partsize"):
        b(A, 0)
    bad = A.copy()
    bad.indices = bad.indices.copy()
    bad.indices[1], bad.indices[2] = bad.indices[2], bad.indices[1]   # unsorted column
    desc = hsb200._HostSparse.__new__(hsb200._HostSparse)
    import ctypes
    ptr = np.ascontiguousarray(bad.indptr, dtype=np.int32)
    idx = np.ascontiguousarray(bad.indices, dtype=np.int32)
    val = np.ascontiguousarray(bad.data)
    d = hsb200._lib.hs_sparse(9, bad.nnz, 0, 0, ptr.ctypes.data, idx.ctypes.data, val.ctypes.data)
    h = ctypes.c_void_p()
    st = hsb200.lib().hs_l1gs_create(ctypes.byref(d), 2, 1, 1.5, 2, 0, 0, 1, 1, None, ctypes.byref(h))
    assert st == hsb200._lib.HS_ERR_ARG


def random_matrix(n, density, seed, sym=False):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=rng, format="csc")
    A.data = rng.uniform(-1, 1, A.nnz)
    if sym:
        A = A + A.T
    A = A + sp.diags(rng.uniform(3, 5, n) + abs(A).sum(axis=1).A.ravel())
    return W._canon(A.tocsc())


CASES = [(1, 37), (2, 40), (3, 100), (5, 101), (8, 777), (12, 1234), (16, 1000), (17, 999), (24, 2000), (31, 700),
         (32, 2048), (32, 1999), (33, 1111), (64, 3000), (100, 2345), (256, 4000)]


@pytest.mark.parametrize("ps,n", CASES)
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
@pytest.mark.parametrize("cache", ["packed", "view"])
def test_random_bitwise_fp64(ps, n, sweep, cache):
    A = random_matrix(n, min(0.5, 12.0 / n), ps * 7 + n)
    x = np.random.default_rng(n).uniform(-1, 1, n)
    for fmt, isSym in (("csc", False), ("csr", False), ("csc", True)):
        M = A.asformat(fmt)
        ref = O.OracleL1GS(M, ps, isSymA=isSym, sweep=sweep, cache=cache)
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
            M, ps, isSymA=isSym, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], order="reference")
        np.testing.assert_array_equal(P.D_DL1, ref.D)
        np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))
        if cache == "packed" and sweep != "backward":
            np.testing.assert_array_equal(P.SLbuffer, ref.SL)
        if cache == "packed" and sweep != "forward":
            np.testing.assert_array_equal(P.SUbuffer, ref.SU)


# One partition holding the whole matrix (partsize = N, the reference's plain
# Gauss-Seidel check, test/test_preconditioners.jl:614-709), partsize > N (a
# single short partition), and matrices of 1 to 7 rows.
SMALL_CASES = [(50, 50), (50, 64), (1, 16), (2, 2), (3, 16), (33, 32), (7, 256)]


@pytest.mark.parametrize("n,ps", SMALL_CASES)
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
@pytest.mark.parametrize("cache", ["packed", "view"])
def test_single_partition_and_tiny_n(n, ps, sweep, cache):
    A = W.poisson_test_matrix(n)
    x = np.random.default_rng(n * 1000 + ps).uniform(-1, 1, n)
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache=cache)
    want = ref.ldiv(x)
    # the reference's order (bitwise), then the library's own choice, which
    # may reorder a row's sum (relative 1e-12, absolute floor 1e-12 max|y|)
    for order in ("reference", None):
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], order=order)
        np.testing.assert_array_equal(P.D_DL1, ref.D)
        got = gpu_apply(P, x)
        if P.order == "reference":
            np.testing.assert_array_equal(got, want)
        else:
            np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


@pytest.mark.parametrize("ps", [2, 8, 16, 32, 33, 64, 130])
@pytest.mark.parametrize("sweep", ["forward", "symmetric"])
@pytest.mark.parametrize("cache", ["packed", "view"])
def test_fp32_and_mixed_bitwise(ps, sweep, cache):
    """FP32 smoother from an FP32 matrix (reference Float32 semantics) and from
    an FP64 matrix (D_Dl1 in FP64, rounded) with FP64 vectors in and out."""
    A = W.poisson2d_matrix(40, eps=0.3)
    x = np.random.default_rng(ps).uniform(-1, 1, A.shape[0])
    b = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=8)
    # FP32 matrix, FP32 vectors
    A32 = A.astype(np.float32)
    ref = O.OracleL1GS(A32, ps, isSymA=True, sweep=sweep, cache=cache)
    P = b(A32, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], order="reference")
    np.testing.assert_array_equal(gpu_apply(P, x.astype(np.float32), torch.float32), ref.ldiv(x.astype(np.float32)))
    # FP64 matrix, FP32 smoother, FP64 vectors
    Pm = b(A, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], precision=np.float32,
           order="reference")
    D64 = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache=cache).D
    np.testing.assert_array_equal(Pm.D_DL1, D64.astype(np.float32))
    y = gpu_apply(Pm, x, torch.float64)
    refm = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache=cache, dtype=np.float32)
    refm.D = D64.astype(np.float32)
    np.testing.assert_array_equal(y, refm.ldiv(x.astype(np.float32)).astype(np.float64))


@pytest.mark.parametrize("ps", [8, 16, 32])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_view_unaligned_vectors(ps, sweep):
    """x and y that start one element past a 16-byte boundary: the view
    kernels' vector loads and stores give way to element accesses."""
    A = W.poisson3d_7pt(14)
    n = A.shape[0]
    x = np.random.default_rng(ps).uniform(-1, 1, n)
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="view").ldiv(x)
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=8)(
        A, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=hsb200.MatrixViewCache())
    for dtype, want in ((torch.float64, ref),):
        xb = torch.zeros(n + 1, dtype=dtype, device="cuda")
        yb = torch.zeros(n + 1, dtype=dtype, device="cuda")
        xb[1:] = dev(x, dtype)
        hsb200.ldiv_(yb[1:], P, xb[1:])
        torch.cuda.synchronize()
        np.testing.assert_array_equal(yb[1:].cpu().numpy(), want)


def test_in_place_apply():
    A = W.poisson3d_7pt(12)
    x = np.random.default_rng(1).uniform(-1, 1, A.shape[0])
    for cache in ("packed", "view"):
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=64, blocks=8)(
            A, 16, isSymA=True, cache_strategy=CACHES[cache])
        xd = dev(x)
        hsb200.ldiv_(xd, P, xd)
        np.testing.assert_array_equal(xd.cpu().numpy(), gpu_apply(P, x))


@pytest.mark.parametrize("ps", [16, 64, 256])
@pytest.mark.parametrize("cache", ["packed", "view"])
def test_poisson3d_bitwise(ps, cache):
    """7-point Poisson (the 128^3 workload's operator) on 48^3, all sweeps."""
    A = W.poisson3d_7pt(48)
    x = W.rhs_uniform(A.shape[0])
    for sweep in ("forward", "backward", "symmetric"):
        ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache=cache)
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache], order="reference")
        np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))


def test_convdiff_nonsym_bitwise():
    """Non-symmetric upwind convection-diffusion (the 96^3 workload's operator) on 40^3."""
    A = W.convdiff3d_upwind(40)
    x = W.rhs_uniform(A.shape[0])
    for cache in ("packed", "view"):
        ref = O.OracleL1GS(A, 16, sweep="forward", cache=cache)
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, 16, sweep=hsb200.ForwardSweep(), cache_strategy=CACHES[cache])
        np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))


def test_full_size_poisson128_packed_symmetric():
    """The 128^3 workload at full size, partsize 16, symmetric packed: bitwise."""
    A = W.poisson3d_7pt(128)
    x = W.rhs_uniform(A.shape[0])
    ref = O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="packed", nchunks=8, chunksize=16384)
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(A, 16, isSymA=True)
    np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))


@pytest.mark.parametrize("ps", [32, 40, 64])
def test_nonfinite_input_rows_layout(ps):
    """Partsize >= 32 streams are padded to whole tiles; the padding is never
    multiplied in, so an inf in x reaches exactly the rows the reference
    reaches (NaN and inf positions equal to the oracle's)."""
    A = W.poisson2d_matrix(30, eps=0.5)
    x = np.random.default_rng(5).uniform(-1, 1, A.shape[0])
    x[ps + 10] = np.inf
    x[3] = np.nan
    for sweep in ("forward", "backward", "symmetric"):
        ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="packed")
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=20)(
            A, ps, isSymA=True, sweep=SWEEPS[sweep], order="reference")
        np.testing.assert_array_equal(gpu_apply(P, x), ref.ldiv(x))


@pytest.mark.parametrize("grid,ps,sweep,cache", [
    ((128, 128, 128), 16, "symmetric", "packed"),   # 4 chunks of whole groups
    ((1, 1500, 1500), 16, "symmetric", "packed"),   # ragged last group
    ((1, 1500, 1500), 40, "forward", "packed"),     # rows layout
    ((128, 128, 128), 16, "symmetric", "view"),
    ((1, 1500, 1500), 64, "backward", "view"),
])
def test_host_apply_chunked_equals_device(grid, ps, sweep, cache):
    """ldiv! on host vectors (the reference's generic path, l1_gauss_seidel.jl:367-384)
    copies x in, applies and copies y out in chunks of whole partition groups on
    overlapping streams; the result is bitwise the device-vector apply."""
    offs = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    A = W._canon(W._stencil_csr(grid, offs, [np.float64(6.0)] + [np.float64(-1.0)] * 6).tocsc(), "csc")
    x = np.random.default_rng(11).uniform(-1, 1, A.shape[0])
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, ps, isSymA=True, sweep=SWEEPS[sweep], cache_strategy=CACHES[cache])
    want = gpu_apply(P, x)
    got = np.empty_like(x)
    hsb200.ldiv_(got, P, x)
    np.testing.assert_array_equal(got, want)
    got2 = np.empty_like(x)
    hsb200.ldiv_(got2, P, x)   # the copy streams and events are reused
    np.testing.assert_array_equal(got2, want)


@pytest.mark.parametrize("cache", ["packed", "view"])
def test_host_apply_pinned_repeated(cache):
    """Page-locked host vectors reused across calls with new contents (the
    handle's copy streams, apply streams and events are reused): every result is
    bitwise the device-vector apply."""
    import ctypes
    A = W.poisson3d_7pt(128)
    n = A.shape[0]
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, 16, isSymA=True, cache_strategy=CACHES[cache])
    xh = torch.empty(n, dtype=torch.float64, pin_memory=True)
    yh = torch.empty(n, dtype=torch.float64, pin_memory=True)
    rng = np.random.default_rng(12)
    for _ in range(3):
        x = rng.uniform(-1, 1, n)
        xh.copy_(torch.from_numpy(x))
        hsb200._lib.check(hsb200.lib().hs_l1gs_apply_host(P.handle, ctypes.c_void_p(xh.data_ptr()),
                                                          ctypes.c_void_p(yh.data_ptr()), hsb200._lib.HS_F64,
                                                          None))
        np.testing.assert_array_equal(yh.numpy(), gpu_apply(P, x))
