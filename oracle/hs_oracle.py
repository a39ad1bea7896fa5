"""Python face of the CPU oracle (oracle/libhsoracle.so) — TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this
module, as the checker.  The product (hybridsmoothers.jl_b200/hsb200 and
libhsb200.so) never imports it.

The C routines restate HybridSmoothers.jl v0.1.4 (citations in
oracle/hs_oracle_tmpl.h).  This module adds the reference's host-side planning
on top of them:

* ``OracleL1GS`` mirrors ``build_l1prec`` / ``_make_sweep_plan``
  (src/l1_gauss_seidel.jl:317-338, :626-843): which arrays row i is read from
  (CSR row; CSC column i when isSymA; the true row of a non-symmetric CSC via
  DiagonalIndices), D_Dl1, the packed SL/SU buffers in the reference layout,
  and ``ldiv`` (:386-396).
* ``OracleChebyshev`` mirrors ``_build_smoother`` and ``smooth!``
  (src/chebyshev.jl:141-183, :258-322).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libhsoracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class SingularException(Exception):
    """Raised where the reference throws LinearAlgebra.SingularException(col).

    ``col`` is 1-based, as in Julia.
    """

    def __init__(self, col):
        super().__init__(f"SingularException({col})")
        self.col = col


def build():
    """Compile oracle/libhsoracle.so with oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        for sfx in ("_f64", "_f32"):
            getattr(L, "hso_packed_size" + sfx).restype = C.c_int64
            getattr(L, "hso_packed_size" + sfx).argtypes = [C.c_int32, C.c_int32]
            getattr(L, "hso_diag_indices" + sfx).restype = C.c_int32
            getattr(L, "hso_power_rho" + sfx).restype = C.c_double
            getattr(L, "hso_cheb1_astar" + sfx).restype = C.c_double
            getattr(L, "hso_cheb1_astar" + sfx).argtypes = [C.c_int32]
        L.hso_pcg.restype = C.c_int32
        L.hso_gmres.restype = C.c_int32
        L.hso_cg_kjl.restype = C.c_int32
        L.hso_gmres_kjl.restype = C.c_int32
        L.hso_omp_max_threads.restype = C.c_int32
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_vp) if a is not None else None


def _sfx(dtype):
    return "_f64" if np.dtype(dtype) == np.float64 else "_f32"


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def omp_threads():
    return int(lib().hso_omp_max_threads())


def set_threads(t):
    lib().hso_omp_set_threads(C.c_int32(int(t)))


def packed_size(n, ps, dtype=np.float64):
    return int(getattr(lib(), "hso_packed_size" + _sfx(dtype))(n, ps))


def nparts_of(n, ps):
    return -(-n // ps)


# --------------------------------------------------------------------------
# Low-level wrappers
# --------------------------------------------------------------------------

def diag_indices(colptr, rowval, nzval):
    """DiagonalIndices(A) (src/l1_gauss_seidel.jl:422-436), 0-based positions."""
    n = len(colptr) - 1
    diag = np.empty(n, dtype=np.int32)
    f = getattr(lib(), "hso_diag_indices" + _sfx(nzval.dtype))
    r = f(C.c_int32(n), _p(_i32(colptr)), _p(_i32(rowval)), _p(np.ascontiguousarray(nzval)), _p(diag))
    if r >= 0:
        raise SingularException(int(r) + 1)
    return diag


def setup_rowwise(rp, ci, v, ps, eta=1.5, lower=True, upper=True, nchunks=1, chunksize=1):
    """D_Dl1 plus SL/SU in the reference layout from a row-wise matrix."""
    rp, ci, v = _i32(rp), _i32(ci), np.ascontiguousarray(v)
    n = len(rp) - 1
    S = packed_size(n, ps, v.dtype)
    D = np.zeros(n, dtype=v.dtype)
    SL = np.zeros(S, dtype=v.dtype) if lower else None
    SU = np.zeros(S, dtype=v.dtype) if upper else None
    f = getattr(lib(), "hso_l1gs_setup_rowwise" + _sfx(v.dtype))
    f(C.c_int32(n), _p(rp), _p(ci), _p(v), C.c_int32(ps), C.c_double(eta), C.c_int32(nchunks),
      C.c_int32(chunksize), _p(D), _p(SL), _p(SU))
    return D, SL, SU


def dl1_rowwise(rp, ci, v, ps, eta=1.5, nchunks=1, chunksize=1):
    rp, ci, v = _i32(rp), _i32(ci), np.ascontiguousarray(v)
    n = len(rp) - 1
    D = np.zeros(n, dtype=v.dtype)
    getattr(lib(), "hso_dl1_rowwise" + _sfx(v.dtype))(
        C.c_int32(n), _p(rp), _p(ci), _p(v), C.c_int32(ps), C.c_double(eta), C.c_int32(nchunks),
        C.c_int32(chunksize), _p(D))
    return D


def dl1_csc_nonsym_literal(colptr, rowval, nzval, diag, ps, eta=1.5):
    colptr, rowval, nzval, diag = _i32(colptr), _i32(rowval), np.ascontiguousarray(nzval), _i32(diag)
    n = len(colptr) - 1
    D = np.zeros(n, dtype=nzval.dtype)
    getattr(lib(), "hso_dl1_csc_nonsym_literal" + _sfx(nzval.dtype))(
        C.c_int32(n), _p(colptr), _p(rowval), _p(nzval), _p(diag), C.c_int32(ps), C.c_double(eta), _p(D))
    return D


def pack_csc_nonsym(colptr, rowval, nzval, ps, lower):
    colptr, rowval, nzval = _i32(colptr), _i32(rowval), np.ascontiguousarray(nzval)
    n = len(colptr) - 1
    out = np.zeros(packed_size(n, ps, nzval.dtype), dtype=nzval.dtype)
    name = "hso_pack_lower_csc_nonsym" if lower else "hso_pack_upper_csc_nonsym"
    getattr(lib(), name + _sfx(nzval.dtype))(C.c_int32(n), _p(colptr), _p(rowval), _p(nzval),
                                             C.c_int32(ps), _p(out))
    return out


SWEEPS = {"forward": 0, "backward": 1, "symmetric": 2}
KIND_PACKED, KIND_ROWWISE, KIND_CSC_NONSYM = 0, 1, 2


def l1gs_apply(n, ps, sweep, kind, D, x, SL=None, SU=None, rp=None, ci=None, v=None, diag=None,
               nchunks=1, chunksize=1, out=None):
    """ldiv!(y, P, x) for the three storage kinds; returns y."""
    D = np.ascontiguousarray(D)
    x = np.ascontiguousarray(x, dtype=D.dtype)
    y = out if out is not None else np.empty_like(x)
    f = getattr(lib(), "hso_l1gs_apply" + _sfx(D.dtype))
    f(C.c_int32(n), C.c_int32(ps), C.c_int32(sweep), C.c_int32(kind), _p(SL), _p(SU),
      _p(_i32(rp) if rp is not None else None), _p(_i32(ci) if ci is not None else None),
      _p(v), _p(_i32(diag) if diag is not None else None), _p(D), _p(x), _p(y),
      C.c_int32(nchunks), C.c_int32(chunksize))
    return y


def l1_rowsum_csc(colptr, rowval, nzval):
    n = len(colptr) - 1
    out = np.zeros(n, dtype=nzval.dtype)
    getattr(lib(), "hso_l1_rowsum_csc" + _sfx(nzval.dtype))(
        C.c_int32(n), _p(_i32(colptr)), _p(_i32(rowval)), _p(np.ascontiguousarray(nzval)), _p(out))
    return out


def spmv(rp, ci, v, x):
    n = len(rp) - 1
    y = np.empty(n, dtype=v.dtype)
    getattr(lib(), "hso_spmv" + _sfx(v.dtype))(C.c_int32(n), _p(_i32(rp)), _p(_i32(ci)), _p(v),
                                              _p(np.ascontiguousarray(x, dtype=v.dtype)), _p(y))
    return y


def spmv_sub(rp, ci, v, z, r):
    """r = r - A z term by term (five-argument mul!, alpha=-1, beta=1); r updated in place."""
    n = len(rp) - 1
    getattr(lib(), "hso_spmv_sub" + _sfx(v.dtype))(C.c_int32(n), _p(_i32(rp)), _p(_i32(ci)), _p(v),
                                                  _p(np.ascontiguousarray(z, dtype=v.dtype)), _p(r))
    return r


def power_rho(rp, ci, v, l1inv, iters=50):
    n = len(rp) - 1
    wv = np.empty(n, dtype=v.dtype)
    ww = np.empty(n, dtype=v.dtype)
    f = getattr(lib(), "hso_power_rho" + _sfx(v.dtype))
    return float(f(C.c_int32(n), _p(_i32(rp)), _p(_i32(ci)), _p(v), _p(l1inv), C.c_int32(iters),
                   _p(wv), _p(ww)))


def cheb1_astar(k):
    return float(lib().hso_cheb1_astar_f64(int(k)))


def cheb4_smooth(rp, ci, v, l1inv, rho, degree, x, b):
    n = len(rp) - 1
    r = np.zeros(n, dtype=v.dtype)
    z = np.zeros(n, dtype=v.dtype)
    getattr(lib(), "hso_cheb4_smooth" + _sfx(v.dtype))(
        C.c_int32(n), _p(_i32(rp)), _p(_i32(ci)), _p(v), _p(l1inv), C.c_double(rho),
        C.c_int32(degree), _p(x), _p(np.ascontiguousarray(b, dtype=v.dtype)), _p(r), _p(z))
    return x


def cheb1_smooth(rp, ci, v, l1inv, rho, astar, degree, x, b):
    n = len(rp) - 1
    r = np.zeros(n, dtype=v.dtype)
    z = np.zeros(n, dtype=v.dtype)
    t = np.zeros(n, dtype=v.dtype)
    getattr(lib(), "hso_cheb1_smooth" + _sfx(v.dtype))(
        C.c_int32(n), _p(_i32(rp)), _p(_i32(ci)), _p(v), _p(l1inv), C.c_double(rho),
        C.c_double(astar), C.c_int32(degree), _p(x), _p(np.ascontiguousarray(b, dtype=v.dtype)),
        _p(r), _p(z), _p(t))
    return x


# --------------------------------------------------------------------------
# Reference-shaped planning
# --------------------------------------------------------------------------

def materialize_symmetric(A_tri, uplo="U"):
    """get_data(::Symmetric) (src/l1_gauss_seidel.jl:602-610)."""
    tri = sp.triu(A_tri) if uplo == "U" else sp.tril(A_tri)
    full = tri + tri.T - sp.diags(tri.diagonal())
    return full.tocsc() if sp.isspmatrix_csc(A_tri) or A_tri.format == "csc" else full.tocsr()


class OracleL1GS:
    """The reference's L1GSPreconditioner, restated on the CPU.

    A: scipy CSC (SparseMatrixCSC) or CSR (SparseMatrixCSR) matrix.
    sweep: "forward" | "backward" | "symmetric"; cache: "packed" | "view".
    chunks/chunksize mirror BlockPartitioning (only the iteration order changes).
    """

    def __init__(self, A, partsize, isSymA=False, eta=1.5, sweep="symmetric", cache="packed",
                 nchunks=1, chunksize=1, dtype=None):
        if partsize == 0:
            raise ValueError("partsize must be greater than 0")
        fmt = A.format
        if fmt not in ("csc", "csr"):
            raise TypeError("A must be CSC or CSR")
        A = A.copy()
        A.sort_indices()
        if dtype is not None:
            A = A.astype(dtype)
        self.n = A.shape[0]
        self.ps = int(partsize)
        self.sweep = sweep
        self.cache = cache
        self.nchunks, self.chunksize = nchunks, chunksize
        self.dtype = A.dtype
        v = np.ascontiguousarray(A.data)
        ptr, idx = _i32(A.indptr), _i32(A.indices)
        self.diag = None
        lower = sweep in ("forward", "symmetric")
        upper = sweep in ("backward", "symmetric")
        if fmt == "csc" and not isSymA:
            # Non-symmetric CSC: DiagonalIndices (:619), D_Dl1 from the true rows
            # (same ascending-column order as :1135-1216), packing per :1279-1469.
            self.diag = diag_indices(ptr, idx, v)
            T = A.tocsr()
            T.sort_indices()
            self.D = dl1_rowwise(T.indptr, T.indices, T.data, self.ps, eta, nchunks, chunksize)
            self.SL = pack_csc_nonsym(ptr, idx, v, self.ps, True) if (cache == "packed" and lower) else None
            self.SU = pack_csc_nonsym(ptr, idx, v, self.ps, False) if (cache == "packed" and upper) else None
            self.kind = KIND_PACKED if cache == "packed" else KIND_CSC_NONSYM
            self.rp, self.ci, self.v = ptr, idx, v
        else:
            # CSR (any symmetry) or symmetric CSC: row i is read from the stored
            # row (CSR) or column i (CSC), :1101-1129, :1248-1277, :1380-1413.
            D, SL, SU = setup_rowwise(ptr, idx, v, self.ps, eta, lower and cache == "packed",
                                      upper and cache == "packed", nchunks, chunksize)
            self.D, self.SL, self.SU = D, SL, SU
            self.kind = KIND_PACKED if cache == "packed" else KIND_ROWWISE
            self.rp, self.ci, self.v = ptr, idx, v

    def ldiv(self, x, out=None):
        return l1gs_apply(self.n, self.ps, SWEEPS[self.sweep], self.kind, self.D, x, self.SL, self.SU,
                          self.rp, self.ci, self.v, self.diag, self.nchunks, self.chunksize, out)


class OracleChebyshev:
    """_build_smoother + smooth! (src/chebyshev.jl:141-183, :258-322).

    Setup (l1 row sums, rho, a*) is FP64 from the FP64 CSC matrix; ``dtype``
    selects the smoother arithmetic (float64: the reference; float32: FP32
    vectors and matrix with FP64 scalars).  ``rho`` may be given to evaluate
    the recurrence at a fixed spectral estimate.
    """

    def __init__(self, A_csc, kind=4, degree=4, dtype=np.float64, rho=None, power_iters=50):
        A = A_csc.tocsc().astype(np.float64)
        A.sort_indices()
        l1 = l1_rowsum_csc(A.indptr, A.indices, A.data)
        l1inv64 = 1.0 / l1
        Acsr = A.tocsr()
        Acsr.sort_indices()
        self.rho = power_rho(Acsr.indptr, Acsr.indices, Acsr.data, l1inv64, power_iters) if rho is None else float(rho)
        self.kind = kind
        self.degree = degree
        self.a = cheb1_astar(degree) if kind == 1 else None
        self.dtype = np.dtype(dtype)
        self.rp, self.ci = _i32(Acsr.indptr), _i32(Acsr.indices)
        self.v = np.ascontiguousarray(Acsr.data.astype(dtype))
        self.l1inv = np.ascontiguousarray(l1inv64.astype(dtype))
        self.n = A.shape[0]

    def smooth(self, x, b):
        x = np.ascontiguousarray(x, dtype=self.dtype)
        if self.kind == 4:
            return cheb4_smooth(self.rp, self.ci, self.v, self.l1inv, self.rho, self.degree, x, b)
        return cheb1_smooth(self.rp, self.ci, self.v, self.l1inv, self.rho, self.a, self.degree, x, b)

    def apply(self, r):
        """z = M^-1 r with M^-1 := smooth!(0, S, r) (used as a PCG preconditioner)."""
        return self.smooth(np.zeros(self.n, dtype=self.dtype), r)


# --------------------------------------------------------------------------
# Krylov drivers
# --------------------------------------------------------------------------

class _Prec(C.Structure):
    _fields_ = [("type", C.c_int32), ("fp32", C.c_int32), ("ps", C.c_int32), ("sweep", C.c_int32),
                ("kind", C.c_int32), ("SL", _vp), ("SU", _vp), ("D", _vp), ("rp", _vp), ("ci", _vp),
                ("v", _vp), ("diag", _vp), ("l1inv", _vp), ("rho", C.c_double),
                ("astar", C.c_double), ("degree", C.c_int32)]


def _prec_struct(P):
    s = _Prec()
    keep = []
    if P is None:
        s.type = 0
        return s, keep
    if isinstance(P, OracleL1GS):
        s.type = 1
        s.fp32 = int(P.dtype == np.float32)
        s.ps, s.sweep, s.kind = P.ps, SWEEPS[P.sweep], P.kind
        for name in ("SL", "SU", "D", "rp", "ci", "v", "diag"):
            a = getattr(P, name)
            keep.append(a)
            setattr(s, name, _p(a))
    else:
        s.type = 2 if P.kind == 4 else 3
        s.fp32 = int(P.dtype == np.float32)
        s.rp, s.ci, s.v, s.l1inv = _p(P.rp), _p(P.ci), _p(P.v), _p(P.l1inv)
        keep += [P.rp, P.ci, P.v, P.l1inv]
        s.rho = P.rho
        s.astar = P.a if P.a is not None else 0.0
        s.degree = P.degree
    return s, keep


def pcg(A, b, P=None, rtol=1e-8, maxit=10000):
    """Returns (x, iterations or -1, true relative residual)."""
    Ar = A.tocsr().astype(np.float64)
    Ar.sort_indices()
    n = Ar.shape[0]
    x = np.zeros(n)
    rel = C.c_double()
    s, keep = _prec_struct(P)
    it = lib().hso_pcg(C.c_int32(n), _p(_i32(Ar.indptr)), _p(_i32(Ar.indices)), _p(Ar.data),
                       _p(np.ascontiguousarray(b, dtype=np.float64)), _p(x), C.byref(s),
                       C.c_double(rtol), C.c_int32(maxit), C.byref(rel))
    return x, int(it), float(rel.value)


def gmres(A, b, P=None, m=30, rtol=1e-8, maxit=10000):
    Ar = A.tocsr().astype(np.float64)
    Ar.sort_indices()
    n = Ar.shape[0]
    x = np.zeros(n)
    rel = C.c_double()
    s, keep = _prec_struct(P)
    it = lib().hso_gmres(C.c_int32(n), _p(_i32(Ar.indptr)), _p(_i32(Ar.indices)), _p(Ar.data),
                         _p(np.ascontiguousarray(b, dtype=np.float64)), _p(x), C.byref(s),
                         C.c_int32(m), C.c_double(rtol), C.c_int32(maxit), C.byref(rel))
    return x, int(it), float(rel.value)


def cg_krylovjl(A, b, P=None, atol=0.0, rtol=1e-8, itmax=0):
    """Krylov.jl's cg (M = P applied with ldiv!), restated in
    hs_oracle.c:hso_cg_kjl.  Returns (x, niter or -1, true relative residual,
    final preconditioned residual norm)."""
    Ar = A.tocsr().astype(np.float64)
    Ar.sort_indices()
    n = Ar.shape[0]
    x = np.zeros(n)
    rel, rn = C.c_double(), C.c_double()
    s, keep = _prec_struct(P)
    it = lib().hso_cg_kjl(C.c_int32(n), _p(_i32(Ar.indptr)), _p(_i32(Ar.indices)), _p(Ar.data),
                          _p(np.ascontiguousarray(b, dtype=np.float64)), _p(x), C.byref(s), C.c_double(atol),
                          C.c_double(rtol), C.c_int32(itmax), C.byref(rel), C.byref(rn))
    return x, int(it), float(rel.value), float(rn.value)


def gmres_krylovjl(A, b, P=None, memory=30, atol=0.0, rtol=1e-8, itmax=0):
    """Krylov.jl's gmres with restart (memory = restart length) and left
    preconditioner M = P (as LinearSolve passes Pl), restated in
    hs_oracle.c:hso_gmres_kjl.  Returns (x, niter or -1, true relative
    residual, final residual estimate)."""
    Ar = A.tocsr().astype(np.float64)
    Ar.sort_indices()
    n = Ar.shape[0]
    x = np.zeros(n)
    rel, rn = C.c_double(), C.c_double()
    s, keep = _prec_struct(P)
    it = lib().hso_gmres_kjl(C.c_int32(n), _p(_i32(Ar.indptr)), _p(_i32(Ar.indices)), _p(Ar.data),
                             _p(np.ascontiguousarray(b, dtype=np.float64)), _p(x), C.byref(s), C.c_int32(memory),
                             C.c_double(atol), C.c_double(rtol), C.c_int32(itmax), C.byref(rel), C.byref(rn))
    return x, int(it), float(rel.value), float(rn.value)


def amg_richardson(A, P, x, b, sweeps=2):
    """AMG.smooth!(x, s::HybridSmoother, b) (ext/HybridSmoothersAMGExt.jl:26-33):
    `sweeps` times residual = A x (three-argument mul!, row sums in ascending
    column order from zero), residual .-= b, correction = P \\ residual,
    x .-= correction.  P is an OracleL1GS of A; returns the new x."""
    R = A.tocsr()
    R.sort_indices()
    dt = np.dtype(P.dtype)
    v = np.ascontiguousarray(R.data.astype(dt))
    x = np.array(x, dtype=dt)
    b = np.ascontiguousarray(b, dtype=dt)
    for _ in range(sweeps):
        r = spmv(R.indptr, R.indices, v, x)
        r = r - b
        z = P.ldiv(r)
        x = x - z
    return x
