"""Pins the CPU oracle against the reference's own known-answer tests.

Mirrors test/test_preconditioners.jl ("Algorithm", "eta parameter",
"Non-Symmetric CSC", "Partsize", "Solution with LinearSolve", "Sanity Checks")
and test/test_chebyshev.jl of HybridSmoothers.jl.  The golden vectors come
from tests/golden/reference_kats.json, extracted from those files by
tests/golden/make_reference_kats.py (each entry records its file:line).
"""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import hs_oracle as O
from hsb200 import workloads as W

KATS = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_kats.json")))


def kat(name):
    return np.array(KATS[name]["value"])


def cpu_partitioning(n, ps, chunks):
    """_blockpartitioning for KA.CPU (src/l1_gauss_seidel.jl:340-351)."""
    nparts = -(-n // ps)
    return chunks, -(-nparts // chunks)


def gpu_partitioning(n, ps, threads, blocks):
    """_blockpartitioning for KA.GPU (src/l1_gauss_seidel.jl:353-365)."""
    nparts = -(-n // ps)
    chunksize = -(-nparts // blocks)
    return blocks, min(chunksize, threads)


SWEEP_KAT = {"forward": "y_exp_fwd", "backward": "y_exp_bwd", "symmetric": "y_exp_sym"}


@pytest.mark.parametrize("fmt", ["csc", "csr"])
@pytest.mark.parametrize("cache", ["packed", "view"])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_algorithm_kat_cpu_chunks(fmt, cache, sweep):
    """test_sym_result over chunks 1..8 (test/test_preconditioners.jl:16-46, :108-276)."""
    A = W.poisson_test_matrix(9).asformat(fmt)
    x = np.arange(9, dtype=np.float64)
    for chunks in range(1, 9):
        nc, cs = cpu_partitioning(9, 2, chunks)
        P = O.OracleL1GS(A, 2, isSymA=True, sweep=sweep, cache=cache, nchunks=nc, chunksize=cs)
        np.testing.assert_array_equal(P.D, kat("D_Dl1_exp"))
        if cache == "packed":
            if sweep in ("forward", "symmetric"):
                np.testing.assert_array_equal(P.SL, kat("SLbuffer_exp"))
            if sweep in ("backward", "symmetric"):
                np.testing.assert_array_equal(P.SU, kat("SUbuffer_exp"))
        np.testing.assert_allclose(P.ldiv(x), kat(SWEEP_KAT[sweep]), rtol=0, atol=1e-15)


@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_algorithm_kat_gpu_layouts(sweep):
    """Result invariant to blocks x threads in 1..10 (test/gpu/gpu.jl:21-61, :113-357)."""
    A = W.poisson_test_matrix(9)
    x = np.arange(9, dtype=np.float64)
    ref = kat("gpu_" + SWEEP_KAT[sweep])
    for blocks in range(1, 11):
        for threads in range(1, 11):
            nc, cs = gpu_partitioning(9, 2, threads, blocks)
            for cache in ("packed", "view"):
                P = O.OracleL1GS(A, 2, isSymA=True, sweep=sweep, cache=cache, nchunks=nc, chunksize=cs)
                np.testing.assert_allclose(P.ldiv(x), ref, rtol=0, atol=1e-15)


def test_symmetric_wrapper_kat():
    """A Symmetric(...) input is materialised (src/l1_gauss_seidel.jl:602-610)."""
    A = W.poisson_test_matrix(9)
    full = O.materialize_symmetric(sp.triu(A).tocsc(), "U")
    assert abs(full - A).max() == 0
    full = O.materialize_symmetric(sp.tril(A).tocsc(), "L")
    assert abs(full - A).max() == 0


def test_eta_parameter():
    """test/test_preconditioners.jl:278-317."""
    A = W.poisson_test_matrix(9)
    x = np.arange(9, dtype=np.float64)
    for eta, dkey in ((2.0, "D_Dl1_exp"), (3.0, "D_Dl1_eta3"), (1.0, "D_Dl1_exp")):
        # the reference builds without isSymA here: the non-symmetric CSC path
        P = O.OracleL1GS(A, 2, eta=eta, sweep="forward", cache="packed")
        np.testing.assert_array_equal(P.D, kat(dkey))
        np.testing.assert_array_equal(P.SL, kat("SLbuffer_exp"))
    P = O.OracleL1GS(A, 2, eta=2.0, sweep="forward", cache="packed")
    np.testing.assert_allclose(P.ldiv(x), kat("y_exp_fwd"), atol=1e-15, rtol=0)


def _A2():
    A = W.poisson_test_matrix(9).tolil()
    A[0, 7] = -1.0   # A2[1, 8] in the reference (1-based)
    A[1, 7] = -1.0   # A2[2, 8]
    return W._canon(A.tocsc())


@pytest.mark.parametrize("cache", ["packed", "view"])
def test_nonsymmetric_csc(cache):
    """test/test_preconditioners.jl:320-353."""
    A2 = _A2()
    x = np.arange(9, dtype=np.float64)
    P = O.OracleL1GS(A2, 2, sweep="forward", cache=cache)
    np.testing.assert_array_equal(P.D, kat("D_Dl1_exp2"))
    if cache == "packed":
        np.testing.assert_array_equal(P.SL, kat("SLbuffer_exp"))
    np.testing.assert_allclose(P.ldiv(x), kat("y2_fwd_exp"), atol=1e-15, rtol=0)
    P = O.OracleL1GS(A2, 2, sweep="backward", cache=cache)
    np.testing.assert_array_equal(P.D, kat("D_Dl1_exp2"))
    if cache == "packed":
        np.testing.assert_array_equal(P.SU, kat("SUbuffer_exp"))
    np.testing.assert_allclose(P.ldiv(x), kat("y2_bwd_exp"), atol=1e-15, rtol=0)


def test_partsize3_packed_layout():
    """Stored zeros in the packed layout, partsize 3 (test/test_preconditioners.jl:355-364)."""
    A = W.poisson_test_matrix(9)
    P = O.OracleL1GS(A, 3, sweep="forward", cache="packed", nchunks=2, chunksize=2)
    np.testing.assert_array_equal(P.D, kat("D_Dl1_exp"))
    np.testing.assert_array_equal(P.SL, kat("SLbuffer_exp_ps3"))


def test_singular_diagonal_raises():
    """DiagonalIndices throws SingularException on a zero diagonal (src/l1_gauss_seidel.jl:429-430)."""
    A = W.poisson_test_matrix(5).tolil()
    A[2, 2] = 0.0
    A = A.tocsc()   # the explicit zero stays stored
    with pytest.raises(O.SingularException) as e:
        O.OracleL1GS(A, 2, sweep="forward", cache="packed")
    assert e.value.col == 3


def _random_nonsym(n, density, seed):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=rng, format="csc")
    A = A + sp.diags(rng.uniform(2, 4, n)) * (1 + A.sum(axis=1).A.ravel().max())
    A.data = np.where(rng.random(A.nnz) < 0.5, -1, 1) * A.data
    A = A + sp.diags(np.full(n, 10.0))
    return W._canon(A.tocsc())


@pytest.mark.parametrize("ps", [1, 3, 7, 16])
def test_nonsym_literal_matches_rowwise(ps):
    """The O(nnz) D_Dl1 (row scan of the transpose) equals the literal O(N^2)
    binary-search restatement bit for bit, and the CSC packing equals the
    row-wise packing of the transposed matrix."""
    A = _random_nonsym(61, 0.15, ps)
    diag = O.diag_indices(A.indptr, A.indices, A.data)
    lit = O.dl1_csc_nonsym_literal(A.indptr, A.indices, A.data, diag, ps, 1.5)
    T = A.tocsr()
    T.sort_indices()
    row = O.dl1_rowwise(T.indptr, T.indices, T.data, ps, 1.5)
    np.testing.assert_array_equal(lit, row)
    _, SLr, SUr = O.setup_rowwise(T.indptr, T.indices, T.data, ps, 1.5)
    np.testing.assert_array_equal(O.pack_csc_nonsym(A.indptr, A.indices, A.data, ps, True), SLr)
    np.testing.assert_array_equal(O.pack_csc_nonsym(A.indptr, A.indices, A.data, ps, False), SUr)


@pytest.mark.parametrize("ps", [1, 2, 5, 16, 33])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_packed_view_bitwise(ps, sweep):
    """Every accumulation is in ascending column order, so packed, row-wise view
    and the non-symmetric CSC binary search agree bit for bit (the packed
    buffer only adds +0.0 terms)."""
    A = _random_nonsym(97, 0.08, 7 + ps)
    x = np.random.default_rng(ps).uniform(-1, 1, A.shape[0])
    yp = O.OracleL1GS(A, ps, sweep=sweep, cache="packed").ldiv(x)
    yv = O.OracleL1GS(A, ps, sweep=sweep, cache="view").ldiv(x)
    yr = O.OracleL1GS(A.tocsr(), ps, sweep=sweep, cache="view").ldiv(x)
    yq = O.OracleL1GS(A.tocsr(), ps, sweep=sweep, cache="packed").ldiv(x)
    np.testing.assert_array_equal(yp, yv)
    np.testing.assert_array_equal(yp, yr)
    np.testing.assert_array_equal(yp, yq)


def test_symmetric_is_bwd_of_scaled_fwd():
    """Symmetric = backward(D_Dl1 .* forward(x)) (src/l1_gauss_seidel.jl:880-906)."""
    A = W.poisson2d_matrix(12, 0.3)
    x = np.random.default_rng(3).uniform(-1, 1, A.shape[0])
    f = O.OracleL1GS(A, 5, isSymA=True, sweep="forward", cache="packed")
    b = O.OracleL1GS(A, 5, isSymA=True, sweep="backward", cache="packed")
    s = O.OracleL1GS(A, 5, isSymA=True, sweep="symmetric", cache="packed")
    np.testing.assert_array_equal(s.ldiv(x), b.ldiv(f.D * f.ldiv(x)))


# ---------------------------------------------------------------------------
# Solver integration (test/test_preconditioners.jl:366-533), own Krylov drivers
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("cache", ["packed", "view"])
@pytest.mark.parametrize("sweep", ["forward", "backward"])
def test_gmres_convection_diffusion(cache, sweep):
    A = W.convection_diffusion_matrix(60, eps=0.1)
    b = np.ones(A.shape[0])
    _, it0, rel0 = O.gmres(A, b, None, rtol=1e-8)
    P = O.OracleL1GS(A, 10, sweep=sweep, cache=cache)
    x, it, rel = O.gmres(A, b, P, rtol=1e-8)
    assert it0 > 0 and it > 0
    assert rel <= 1e-8 * 1.01
    assert it <= it0


@pytest.mark.parametrize("cache", ["packed", "view"])
def test_pcg_poisson2d_symmetric(cache):
    A = W.poisson2d_matrix(100, eps=0.1)
    b = np.ones(A.shape[0])
    _, it0, _ = O.pcg(A, b, None, rtol=1e-8)
    P = O.OracleL1GS(A, 10, isSymA=True, sweep="symmetric", cache=cache)
    x, it, rel = O.pcg(A, b, P, rtol=1e-8)
    assert 0 < it <= it0
    assert rel < 1e-7


@pytest.mark.parametrize("cache", ["packed", "view"])
@pytest.mark.parametrize("sweep", ["forward", "backward"])
def test_gmres_poisson2d(cache, sweep):
    A = W.poisson2d_matrix(100, eps=0.1)
    b = np.ones(A.shape[0])
    _, it0, _ = O.gmres(A, b, None, rtol=1e-8)
    P = O.OracleL1GS(A, 10, isSymA=True, sweep=sweep, cache=cache)
    _, it, rel = O.gmres(A, b, P, rtol=1e-8)
    assert 0 < it <= it0 and rel <= 1.01e-8


def test_pcg_symmetric_wrapper():
    A = O.materialize_symmetric(sp.triu(W.poisson2d_matrix(120, eps=0.1)).tocsc())
    b = np.ones(A.shape[0])
    _, it0, _ = O.pcg(A, b, None, rtol=1e-8)
    for cache in ("packed", "view"):
        P = O.OracleL1GS(A, 10, isSymA=True, sweep="symmetric", cache=cache)
        _, it, _ = O.pcg(A, b, P, rtol=1e-8)
        assert 0 < it <= it0


# ---------------------------------------------------------------------------
# Sanity checks (test/test_preconditioners.jl:534-710)
# ---------------------------------------------------------------------------

def test_sparse_l1gs_as_gauss_seidel():
    """partsize = N makes L1GS plain Gauss-Seidel: fwd and bwd need the same
    number of stationary iterations, symmetric about half (+-1%)."""
    N = 50
    A = W.poisson_test_matrix(N)
    b = np.ones(N)
    L = sp.tril(A, -1).tocsr()
    U = sp.triu(A, 1).tocsr()
    Pf = O.OracleL1GS(A, N, isSymA=True, sweep="forward", cache="view")
    Pb = O.OracleL1GS(A, N, isSymA=True, sweep="backward", cache="view")

    def run(step):
        x = np.zeros(N)
        for it in range(1, 10001):
            x = step(x)
            if np.linalg.norm(A @ x - b) < 1e-10:
                return it
        return 10000

    it_f = run(lambda x: Pf.ldiv(b - U @ x))
    it_b = run(lambda x: Pb.ldiv(b - L @ x))
    it_s = run(lambda x: Pb.ldiv(b - L @ Pf.ldiv(b - U @ x)))
    assert it_f == it_b
    assert abs(it_s - it_f // 2) <= it_f // 100


# ---------------------------------------------------------------------------
# Chebyshev (test/test_chebyshev.jl)
# ---------------------------------------------------------------------------

def test_l1_rowsum_kat():
    A = W.poisson_test_matrix(5)
    np.testing.assert_array_equal(O.l1_rowsum_csc(A.indptr, A.indices, A.data), kat("l1_rowsum_poisson5"))


def test_spectral_radius_bounds():
    A = W.poisson_test_matrix(100)
    S = O.OracleChebyshev(A, kind=4)
    assert 0 < S.rho <= 1


def test_astar_table():
    """a* for k = 1..8 against the docstring table (src/chebyshev.jl:208-210), and
    monotonically decreasing (test/test_chebyshev.jl:160-165)."""
    a = np.array([O.cheb1_astar(k) for k in range(1, 9)])
    np.testing.assert_allclose(a, kat("astar_table"), atol=6e-4)
    assert np.all(np.diff(a) < 0)
    assert all(0 < v < 1 for v in a)


@pytest.mark.parametrize("kind", [4, 1])
def test_cheb_reduces_residual(kind):
    N = 300
    A = W.poisson_test_matrix(N)
    b = np.ones(N)
    res = []
    for degree in (1, 2, 4, 8):
        S = O.OracleChebyshev(A, kind=kind, degree=degree)
        x = S.smooth(np.zeros(N), b)
        r = np.linalg.norm(b - A @ x)
        assert r < np.linalg.norm(b)
        res.append(r)
    assert all(res[i] >= res[i + 1] for i in range(3))   # issorted(rev=true)


@pytest.mark.parametrize("kind", [4, 1])
def test_cheb_monotone_over_applications(kind):
    N = 200
    A = W.poisson_test_matrix(N)
    b = np.random.default_rng(42).random(N)
    S = O.OracleChebyshev(A, kind=kind, degree=4)
    x = np.zeros(N)
    prev = np.linalg.norm(b)
    for _ in range(10):
        x = S.smooth(x, b)
        cur = np.linalg.norm(b - A @ x)
        assert cur < prev
        prev = cur
    assert prev / np.linalg.norm(b) < 0.9


def test_cheb_first_vs_fourth_comparable():
    N = 300
    A = W.poisson_test_matrix(N)
    b = np.random.default_rng(7).random(N)
    r0 = np.linalg.norm(b)
    for degree in range(1, 6):
        x4 = O.OracleChebyshev(A, kind=4, degree=degree).smooth(np.zeros(N), b)
        x1 = O.OracleChebyshev(A, kind=1, degree=degree).smooth(np.zeros(N), b)
        r4 = np.linalg.norm(b - A @ x4) / r0
        r1 = np.linalg.norm(b - A @ x1) / r0
        assert r4 < 1 and r1 < 1
        assert abs(r1 - r4) / r4 < 0.02


@pytest.mark.parametrize("kind", [4, 1])
def test_cheb_repeatable(kind):
    N = 500
    A = W.poisson_test_matrix(N)
    S = O.OracleChebyshev(A, kind=kind, degree=4)
    x1 = S.smooth(np.zeros(N), np.ones(N))
    x2 = S.smooth(np.zeros(N), np.ones(N))
    np.testing.assert_array_equal(x1, x2)


@pytest.mark.parametrize("kind", [4, 1])
def test_cheb_as_pcg_preconditioner(kind):
    A = W.poisson2d_matrix(60, eps=0.5)
    b = np.ones(A.shape[0])
    _, it0, _ = O.pcg(A, b, None)
    _, it, rel = O.pcg(A, b, O.OracleChebyshev(A, kind=kind, degree=4))
    assert 0 < it < it0 and rel < 1e-7


def test_fp32_smoother_inside_fp64_pcg():
    A = W.poisson2d_matrix(50, eps=0.5)
    b = np.ones(A.shape[0])
    _, it64, _ = O.pcg(A, b, O.OracleL1GS(A, 10, isSymA=True, sweep="symmetric", cache="packed"))
    _, it32, rel = O.pcg(A, b, O.OracleL1GS(A, 10, isSymA=True, sweep="symmetric", cache="packed",
                                            dtype=np.float32))
    assert rel < 1e-7 and abs(it32 - it64) <= 2
