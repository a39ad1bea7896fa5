"""hsb200 — B200 (sm_100a) implementation of HybridSmoothers.jl's
preconditioner/smoother apply path, behind the reference's own interface.

Host-side mirror of the reference API (names, argument meaning, errors):

  reference (HybridSmoothers.jl v0.1.4)             here
  ------------------------------------------------  -------------------------------------
  L1GSPrecBuilder(backend; threads, blocks)         L1GSPrecBuilder(CUDABackend(), threads=, blocks=)
    (src/l1_gauss_seidel.jl:240-262)
  builder(A, partsize; isSymA, η, sweep,            builder(A, partsize, isSymA=, eta=, sweep=,
          cache_strategy)  (:287-313)                       cache_strategy=, precision=)
  ForwardSweep/BackwardSweep/SymmetricSweep         same names
  PackedBufferCache/MatrixViewCache                 same names
  Symmetric(A) input  (:305-313, :602-610)          Symmetric(A, uplo)
  LinearSolve.ldiv!(y, P, x)  (:367-396)            ldiv_(y, P, x)
  P \\ x  (:398-407)                                 backslash(P, x)
  ChebyshevFourth/First(; degree, backend)          ChebyshevFourth/First(degree=, backend=, eig=)
    (src/chebyshev.jl:115-119, :218-222)
  _build_smoother(cfg, A)  (:141-156, :258-276)     build_smoother(cfg, A)
  smooth!(x, s, b)  (:158-183, :278-322)            smooth_(x, s, b)
  mul!(y, A, x[, α, β])  (SparseMatricesCSR)        mul_(y, A, x, alpha, beta) on DeviceSparseMatrix

Host matrices are scipy.sparse CSC ("SparseMatrixCSC") or CSR
("SparseMatrixCSR") matrices.  Device vectors are torch CUDA tensors; host
vectors are numpy arrays (ldiv_ then copies through the device, like the
reference's generic ldiv!).  There is no CPU backend: KA.CPU() work is not part
of this library and asking for it raises.
"""
from __future__ import annotations

import ctypes as C
from collections import namedtuple

import numpy as np
import scipy.sparse as sp

from . import _lib as _L
from ._lib import HSError, SingularException, check, kernel_launches, lib

__all__ = [
    "CPU", "CUDABackend", "GPUConfig", "CPUConfig", "L1GSPrecBuilder", "L1GSPreconditioner",
    "ForwardSweep", "BackwardSweep", "SymmetricSweep", "PackedBufferCache", "MatrixViewCache",
    "Symmetric", "ldiv_", "backslash", "ChebyshevFourth", "ChebyshevFirst", "build_smoother",
    "smooth_", "DeviceSparseMatrix", "mul_", "pcg", "gmres", "cg_krylovjl", "gmres_krylovjl", "LinearProblem",
    "KrylovJL_CG", "KrylovJL_GMRES", "solve", "HSError", "SingularException", "kernel_launches",
    "BlockPartitioning",
]


# ---------------------------------------------------------------------------
# Backends and device configuration (src/l1_gauss_seidel.jl:185-224)
# ---------------------------------------------------------------------------
class CPU:
    """KA.CPU(): accepted for signature parity, rejected at build (no CPU path here)."""


class CUDABackend:
    """The only backend of this library: a B200 (sm_100a) GPU, device `device`."""

    def __init__(self, device=0):
        self.device = device


class CPUConfig:
    def __init__(self, chunks):
        if chunks <= 0:
            raise ValueError("`chunks` must be greater than 0")
        self.chunks = chunks


class GPUConfig:
    def __init__(self, threads, blocks):
        if threads <= 0:
            raise ValueError("`threads` must be greater than 0")
        if blocks <= 0:
            raise ValueError("`blocks` must be greater than 0")
        self.threads, self.blocks = int(threads), int(blocks)


# ---------------------------------------------------------------------------
# Sweep and cache tags (src/l1_gauss_seidel.jl:11-100)
# ---------------------------------------------------------------------------
class AbstractSweep:
    code = None


class ForwardSweep(AbstractSweep):
    """M = D + L."""
    code = _L.HS_SWEEP_FORWARD


class BackwardSweep(AbstractSweep):
    """M = D + U."""
    code = _L.HS_SWEEP_BACKWARD


class SymmetricSweep(AbstractSweep):
    """M = (D + L) D^-1 (D + U), applied as backward(D .* forward(x))."""
    code = _L.HS_SWEEP_SYMMETRIC


class AbstractCacheStrategy:
    code = None


class PackedBufferCache(AbstractCacheStrategy):
    """Strict triangles of the diagonal blocks packed densely (GPU default)."""
    code = _L.HS_CACHE_PACKED


class MatrixViewCache(AbstractCacheStrategy):
    """Sweeps read the sparse matrix directly."""
    code = _L.HS_CACHE_VIEW


class Symmetric:
    """LinearAlgebra.Symmetric(A, uplo): only the `uplo` triangle of `data` is used."""

    def __init__(self, data, uplo="U"):
        if uplo not in ("U", "L"):
            raise ValueError("uplo must be 'U' or 'L'")
        self.data, self.uplo = data, uplo

    def materialize(self):
        """get_data(::Symmetric) (src/l1_gauss_seidel.jl:602-610): tri + tri' - diag."""
        A = self.data
        tri = sp.triu(A) if self.uplo == "U" else sp.tril(A)
        full = tri + tri.T - sp.diags(tri.diagonal())
        return full.asformat(A.format)


BlockPartitioning = namedtuple("BlockPartitioning", "partsize nparts nchunks chunksize backend")

# ---------------------------------------------------------------------------
# Host matrix marshalling
# ---------------------------------------------------------------------------


def _dtype_code(dt):
    dt = np.dtype(dt)
    if dt == np.float64:
        return _L.HS_F64
    if dt == np.float32:
        return _L.HS_F32
    raise TypeError(f"unsupported value type {dt}")


class _HostSparse:
    """Keeps a canonical (sorted, int32) host copy alive while the C call reads it."""

    def __init__(self, A, dtype=None):
        if not sp.issparse(A):
            raise TypeError("A must be a scipy.sparse CSC or CSR matrix")
        fmt = A.format
        if fmt not in ("csc", "csr"):
            raise TypeError("A must be CSC (SparseMatrixCSC) or CSR (SparseMatrixCSR)")
        if A.shape[0] != A.shape[1]:
            raise ValueError("A must be square")
        if not A.has_canonical_format:
            # sorted, duplicate-free copy; a canonical input is read in place
            A = A.copy()
            A.sort_indices()
            A.sum_duplicates()
        if dtype is not None and A.dtype != np.dtype(dtype):
            A = A.astype(dtype)
        self._A = A
        self.ptr = np.ascontiguousarray(A.indptr, dtype=np.int32)
        self.idx = np.ascontiguousarray(A.indices, dtype=np.int32)
        self.val = np.ascontiguousarray(A.data)
        self.desc = _L.hs_sparse(A.shape[0], A.nnz, _L.HS_CSC if fmt == "csc" else _L.HS_CSR,
                                 _dtype_code(self.val.dtype), self.ptr.ctypes.data, self.idx.ctypes.data,
                                 self.val.ctypes.data)
        self.format = fmt
        self.dtype = self.val.dtype


def _stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev_ptr(t, dtype):
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda):
        raise TypeError("expected a CUDA tensor")
    if t.dtype != dtype or not t.is_contiguous():
        raise TypeError(f"expected a contiguous {dtype} CUDA tensor, got {t.dtype}")
    return C.c_void_p(t.data_ptr())


def _torch_dtype(code):
    import torch
    return torch.float64 if code == _L.HS_F64 else torch.float32


def _io_code(t):
    import torch
    return _L.HS_F64 if t.dtype == torch.float64 else _L.HS_F32


# ---------------------------------------------------------------------------
# L1 Gauss-Seidel
# ---------------------------------------------------------------------------
class L1GSPrecBuilder:
    """L1GSPrecBuilder(backend; threads, blocks) (src/l1_gauss_seidel.jl:240-262)."""

    def __init__(self, backend=None, threads=None, blocks=None, chunks=None, device_config=None):
        backend = backend if backend is not None else CUDABackend()
        if isinstance(backend, CPU):
            self.device_config = device_config or CPUConfig(chunks if chunks is not None else 1)
        else:
            if device_config is None:
                if threads is None or blocks is None:
                    raise TypeError("L1GSPrecBuilder(CUDABackend(); threads, blocks) needs threads and blocks")
                device_config = GPUConfig(threads, blocks)
            self.device_config = device_config
        self.backend = backend

    def _default_partsize(self):
        cfg = self.device_config
        return cfg.chunks if isinstance(cfg, CPUConfig) else cfg.blocks

    def __call__(self, A, partsize=None, isSymA=False, eta=1.5, sweep=None, cache_strategy=None,
                 precision=None, stream=None, threads_per_part=0, order=None):
        """builder(A, partsize; isSymA, η, sweep, cache_strategy) (:287-313).

        precision: None (the matrix type) or np.float32 for an FP32 smoother
        built from an FP64 matrix.
        threads_per_part: 0 (the library chooses), 1 (one thread per
        partition: every row summed in the reference's order, bit-identical),
        8 with a partsize that is a multiple of 8 (the blocked sweep over 8x8
        tiles, the library's choice from partsize 32), or 4/16/32 lanes
        sharing a partition column by column (forward sweeps stay
        bit-identical; backward/symmetric agree to rounding).  Packed caches
        only; a matrix-view cache always uses 1.
        order: None (the library chooses), "reference" (every row summed in
        the reference's order: bit-identical results) or "any" (the library
        may reorder a row's sum: relative 1e-12 of the reference in FP64).
        """
        if isinstance(self.backend, CPU):
            raise NotImplementedError("the KA.CPU() backend is not part of this library (B200 only)")
        partsize = self._default_partsize() if partsize is None else int(partsize)
        if partsize == 0:
            raise ValueError("partsize must be greater than 0")
        sweep = sweep if sweep is not None else SymmetricSweep()
        cache_strategy = cache_strategy if cache_strategy is not None else PackedBufferCache()
        if isinstance(A, Symmetric):
            A = A.materialize()
            isSymA = True
        codes = {None: 0, "reference": 1, "any": 2}
        if order not in codes:
            raise ValueError("order must be None, 'reference' or 'any'")
        return L1GSPreconditioner(self, A, partsize, bool(isSymA), float(eta), sweep, cache_strategy,
                                  precision, stream, int(threads_per_part), codes[order])


class L1GSPreconditioner:
    """L1GSPreconditioner(partitioning, sweep) (src/l1_gauss_seidel.jl:180-183)."""

    def __init__(self, builder, A, partsize, isSymA, eta, sweep, cache, precision, stream, threads_per_part=0,
                 order=0):
        import torch
        hA = _HostSparse(A)
        sdt = _L.HS_F32 if (precision is not None and np.dtype(precision) == np.float32) else hA.desc.dtype
        cfg = builder.device_config
        self._h = C.c_void_p()
        # bound now: module globals may already be gone when __del__ runs at exit
        self._destroy = _L.lib().hs_l1gs_destroy
        torch.cuda.init()
        opts = _L.hs_l1gs_options(int(threads_per_part), int(order))
        check(lib().hs_l1gs_create_opts(C.byref(hA.desc), int(partsize), int(isSymA), float(eta), sweep.code,
                                        cache.code, sdt, cfg.threads, cfg.blocks, C.byref(opts),
                                        _stream_ptr(stream), C.byref(self._h)))
        info = _L.hs_l1gs_info()
        check(lib().hs_l1gs_info_get(self._h, C.byref(info)))
        self.info = info
        self.n = info.n
        self.sweep_tag = sweep
        self.cache_strategy = cache
        self.smoother_dtype = np.float64 if sdt == _L.HS_F64 else np.float32
        self.partitioning = BlockPartitioning(info.partsize, info.nparts, info.nchunks, info.chunksize,
                                              builder.backend)
        self.threads_per_part = info.threads_per_part
        self.order = "reference" if info.order == 1 else "any"

    # -- introspection (P.sweep.op.D_DL1, .L.SLbuffer, .U.SUbuffer) --------
    @property
    def D_DL1(self):
        out = np.empty(self.n, dtype=self.smoother_dtype)
        check(lib().hs_l1gs_get_diag(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    def _packed(self, which):
        out = np.empty(self.info.packed_len, dtype=self.smoother_dtype)
        check(lib().hs_l1gs_get_packed(self._h, which, out.ctypes.data_as(C.c_void_p), out.size))
        return out

    @property
    def SLbuffer(self):
        return self._packed(0)

    @property
    def SUbuffer(self):
        return self._packed(1)

    @property
    def diag_indices(self):
        out = np.empty(self.n, dtype=np.int32)
        check(lib().hs_l1gs_get_diag_indices(self._h, out.ctypes.data_as(C.c_void_p)))
        return out

    @property
    def handle(self):
        return self._h

    def apply(self, x, y, stream=None):
        """y = M^-1 x on device tensors (the C entry point hs_l1gs_apply)."""
        if x.numel() != self.n or y.numel() != self.n:
            raise ValueError("vector length does not match the preconditioner")
        io = _io_code(y)
        check(lib().hs_l1gs_apply(self._h, _dev_ptr(x, _torch_dtype(io)), _dev_ptr(y, _torch_dtype(io)), io,
                                  _stream_ptr(stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h and destroy is not None:
            try:
                destroy(h)
            except Exception:
                pass
            self._h = None

    def __repr__(self):
        return (f"L1GSPreconditioner({type(self.sweep_tag).__name__[:-5]}, CUDABackend, "
                f"nparts={self.partitioning.nparts})")


def ldiv_(y, P, x, stream=None):
    """LinearSolve.ldiv!(y, P, x): y = M^-1 x; returns None.

    torch CUDA tensors go straight to the device kernels; numpy arrays take the
    reference's generic path (copy to the device, sweep, copy back).
    """
    if isinstance(P, _ChebSmoother):
        return P.ldiv_(y, x, stream)
    if isinstance(x, np.ndarray):
        if not isinstance(y, np.ndarray) or y.dtype != x.dtype or x.shape != (P.n,) or y.shape != (P.n,):
            raise ValueError("x and y must be host vectors of the same type and length n")
        xc = np.ascontiguousarray(x)
        if not y.flags.c_contiguous:
            raise ValueError("y must be contiguous")
        io = _dtype_code(x.dtype)
        check(lib().hs_l1gs_apply_host(P.handle, xc.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p), io,
                                       _stream_ptr(stream)))
        return None
    P.apply(x, y, stream)
    return None


def backslash(P, x, stream=None):
    """P \\ x (src/l1_gauss_seidel.jl:398-407): allocates y."""
    if isinstance(x, np.ndarray):
        y = np.empty_like(x)
    else:
        import torch
        y = torch.empty_like(x)
    ldiv_(y, P, x, stream)
    return y


# ---------------------------------------------------------------------------
# Device sparse matrix: mul!
# ---------------------------------------------------------------------------
class DeviceSparseMatrix:
    """A CSR copy of A on the device (SparseMatrixCSR after adapt)."""

    def __init__(self, A, dtype=np.float64, stream=None):
        import torch
        torch.cuda.init()
        hA = _HostSparse(A)
        self.n = hA.desc.n
        self.dtype = np.dtype(dtype)
        self._h = C.c_void_p()
        # bound now: module globals may already be gone when __del__ runs at exit
        self._destroy = _L.lib().hs_matrix_destroy
        check(lib().hs_matrix_create(C.byref(hA.desc), _dtype_code(dtype), _stream_ptr(stream), C.byref(self._h)))

    @property
    def handle(self):
        return self._h

    def __del__(self):
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h and destroy is not None:
            try:
                destroy(h)
            except Exception:
                pass
            self._h = None


def mul_(y, A, x, alpha=1.0, beta=0.0, stream=None):
    """mul!(y, A, x, α, β) on device vectors."""
    td = _torch_dtype(_dtype_code(A.dtype))
    check(lib().hs_matrix_spmv(A.handle, _dev_ptr(x, td), _dev_ptr(y, td), float(alpha), float(beta),
                               _stream_ptr(stream)))


# ---------------------------------------------------------------------------
# Chebyshev smoothers (src/chebyshev.jl)
# ---------------------------------------------------------------------------
class ChebyshevFourth:
    """ChebyshevFourth(; degree = 4, backend) (src/chebyshev.jl:115-119)."""
    kind = 4

    def __init__(self, degree=4, backend=None, eig="power", precision=None):
        self.degree, self.backend, self.eig, self.precision = int(degree), backend or CUDABackend(), eig, precision


class ChebyshevFirst(ChebyshevFourth):
    """ChebyshevFirst(; degree = 4, backend) (src/chebyshev.jl:218-222)."""
    kind = 1


class _ChebSmoother:
    def __init__(self, cfg, A, stream=None):
        import torch
        if isinstance(cfg.backend, CPU):
            raise NotImplementedError("the KA.CPU() backend is not part of this library (B200 only)")
        torch.cuda.init()
        hA = _HostSparse(A.tocsc() if A.format != "csc" else A, dtype=np.float64)
        sdt = _L.HS_F32 if (cfg.precision is not None and np.dtype(cfg.precision) == np.float32) else _L.HS_F64
        eig = _L.HS_EIG_LANCZOS if cfg.eig == "lanczos" else _L.HS_EIG_POWER
        self._h = C.c_void_p()
        # bound now: module globals may already be gone when __del__ runs at exit
        self._destroy = _L.lib().hs_cheb_destroy
        check(lib().hs_cheb_create(C.byref(hA.desc), cfg.kind, cfg.degree, eig, sdt, _stream_ptr(stream),
                                   C.byref(self._h)))
        self.smoother_dtype = np.float64 if sdt == _L.HS_F64 else np.float32
        self.n = hA.desc.n
        self.degree = cfg.degree
        self.kind = cfg.kind

    @property
    def info(self):
        i = _L.hs_cheb_info()
        check(lib().hs_cheb_info_get(self._h, C.byref(i)))
        return i

    @property
    def rho(self):
        return self.info.rho

    @property
    def a(self):
        return self.info.astar

    def set_rho(self, rho):
        check(lib().hs_cheb_set_rho(self._h, float(rho)))

    @property
    def handle(self):
        return self._h

    def ldiv_(self, z, r, stream=None):
        io = _io_code(z)
        check(lib().hs_cheb_apply(self._h, _dev_ptr(r, _torch_dtype(io)), _dev_ptr(z, _torch_dtype(io)), io,
                                  _stream_ptr(stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h and destroy is not None:
            try:
                destroy(h)
            except Exception:
                pass
            self._h = None


def build_smoother(cfg, A, stream=None):
    """_build_smoother(config, A_csc) (src/chebyshev.jl:141-156, :258-276)."""
    return _ChebSmoother(cfg, A, stream)


def smooth_(x, s, b, stream=None):
    """smooth!(x, s, b): x updated in place (device tensors in the smoother type)."""
    td = _torch_dtype(_dtype_code(s.smoother_dtype))
    check(lib().hs_cheb_smooth(s.handle, _dev_ptr(x, td), _dev_ptr(b, td), _stream_ptr(stream)))


# ---------------------------------------------------------------------------
# Krylov drivers
# ---------------------------------------------------------------------------
def _prec_args(P):
    if P is None:
        return _L.HS_PREC_NONE, None
    if isinstance(P, L1GSPreconditioner):
        return _L.HS_PREC_L1GS, P.handle
    if isinstance(P, _ChebSmoother):
        return _L.HS_PREC_CHEB, P.handle
    raise TypeError("unsupported preconditioner")


def pcg(A, b, x, P=None, rtol=1e-8, maxit=10000, stream=None):
    """Preconditioned CG on the device (FP64): returns hs_solve_info."""
    import torch
    t, h = _prec_args(P)
    info = _L.hs_solve_info()
    st = lib().hs_pcg_solve(A.handle, t, h, _dev_ptr(b, torch.float64), _dev_ptr(x, torch.float64), float(rtol),
                            int(maxit), _stream_ptr(stream), C.byref(info))
    if st not in (_L.HS_OK, _L.HS_ERR_NOT_CONVERGED):
        check(st)
    return info


def gmres(A, b, x, P=None, restart=30, rtol=1e-8, maxit=10000, stream=None):
    """Restarted right-preconditioned GMRES on the device (FP64)."""
    import torch
    t, h = _prec_args(P)
    info = _L.hs_solve_info()
    st = lib().hs_gmres_solve(A.handle, t, h, int(restart), _dev_ptr(b, torch.float64), _dev_ptr(x, torch.float64),
                              float(rtol), int(maxit), _stream_ptr(stream), C.byref(info))
    if st not in (_L.HS_OK, _L.HS_ERR_NOT_CONVERGED):
        check(st)
    return info


def cg_krylovjl(A, b, x, P=None, atol=0.0, rtol=1e-8, itmax=0, stream=None):
    """Krylov.jl's cg with M = P applied by ldiv! (FP64, device vectors):
    stops when sqrt(r.z) <= atol + rtol sqrt(r0.z0), z = M^-1 r.  itmax 0 = 2n.
    Returns hs_solve_info (iterations = Krylov.jl's niter)."""
    import torch
    t, h = _prec_args(P)
    info = _L.hs_solve_info()
    st = lib().hs_cg_krylovjl(A.handle, t, h, _dev_ptr(b, torch.float64), _dev_ptr(x, torch.float64), float(atol),
                              float(rtol), int(itmax), _stream_ptr(stream), C.byref(info))
    if st not in (_L.HS_OK, _L.HS_ERR_NOT_CONVERGED):
        check(st)
    return info


def gmres_krylovjl(A, b, x, P=None, memory=30, atol=0.0, rtol=1e-8, itmax=0, stream=None):
    """Krylov.jl's gmres with restart length `memory` and left preconditioner
    M = P (as LinearSolve passes Pl): stops when the estimate of
    ||M^-1 (b - A x)|| is at most atol + rtol ||M^-1 b||.  itmax 0 = 2n."""
    import torch
    t, h = _prec_args(P)
    info = _L.hs_solve_info()
    st = lib().hs_gmres_krylovjl(A.handle, t, h, int(memory), _dev_ptr(b, torch.float64), _dev_ptr(x, torch.float64),
                                 float(atol), float(rtol), int(itmax), _stream_ptr(stream), C.byref(info))
    if st not in (_L.HS_OK, _L.HS_ERR_NOT_CONVERGED):
        check(st)
    return info


# ---------------------------------------------------------------------------
# The caller's interface: LinearSolve.jl's solve(LinearProblem(A, b), alg; Pl)
# (README.md:27-29, test/test_preconditioners.jl:65,93) on the device drivers.
# ---------------------------------------------------------------------------
class LinearProblem:
    """LinearProblem(A, b): A a scipy.sparse CSC/CSR matrix, b a numpy vector."""

    def __init__(self, A, b):
        self.A, self.b = A, np.asarray(b, dtype=np.float64)


class KrylovJL_CG:
    """KrylovJL_CG(): Krylov.jl's cg."""


class KrylovJL_GMRES:
    """KrylovJL_GMRES(; gmres_restart = 0): Krylov.jl's gmres, restarted every
    gmres_restart iterations; 0 (LinearSolve's default) runs without restart,
    here for up to min(n, 1024) iterations (the Krylov basis is allocated up
    front; beyond that it restarts)."""

    def __init__(self, gmres_restart=0):
        if gmres_restart < 0:
            raise ValueError("gmres_restart must be >= 0")
        self.gmres_restart = int(gmres_restart)


class LinearSolution:
    def __init__(self, u, info):
        self.u = u
        self.iters = int(info.iterations)
        self.converged = bool(info.converged)
        self.relres = float(info.relres)
        self.resid = float(info.rnorm)
        self.ms = float(info.ms)


DEFAULT_TOL = float(np.sqrt(np.finfo(np.float64).eps))   # LinearSolve's default abstol and reltol


def solve(prob, alg, Pl=None, abstol=DEFAULT_TOL, reltol=DEFAULT_TOL, maxiters=0, stream=None):
    """solve(prob, alg; Pl, abstol, reltol, maxiters) -> solution with .u (host
    vector) and .iters, on the device: the matrix and b are uploaded, Krylov.jl's
    cg or gmres runs with Pl applied by ldiv! each iteration."""
    import torch
    A = DeviceSparseMatrix(prob.A, stream=stream)
    b = torch.from_numpy(np.ascontiguousarray(prob.b)).cuda()
    x = torch.zeros_like(b)
    if isinstance(alg, KrylovJL_CG):
        info = cg_krylovjl(A, b, x, Pl, atol=abstol, rtol=reltol, itmax=maxiters, stream=stream)
    elif isinstance(alg, KrylovJL_GMRES):
        memory = alg.gmres_restart if alg.gmres_restart > 0 else min(A.n, 1024)
        info = gmres_krylovjl(A, b, x, Pl, memory=memory, atol=abstol, rtol=reltol, itmax=maxiters, stream=stream)
    else:
        raise TypeError("alg must be KrylovJL_CG() or KrylovJL_GMRES()")
    return LinearSolution(x.cpu().numpy(), info)
