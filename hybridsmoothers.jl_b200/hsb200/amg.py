"""The smoothers as algebraic-multigrid smoothers (ext/HybridSmoothersAMGExt.jl).

The reference extends AlgebraicMultigrid.jl: ``AMG.setup_smoother(config, A,
symmetry)`` builds a smoother from a preconditioner builder or a Chebyshev
config, and ``AMG.smooth!(x, s, b)`` applies it on each level.  For an L1GS
builder the smoother is ``HybridSmoother{A, s, residual, correction}``
(:8-13) running two Richardson sweeps per call (:26-33):

    residual = A x;  residual .-= b;  correction = P \\ residual;  x .-= correction

Chebyshev configs are the Chebyshev smoothers themselves (:35-49).

Here the Richardson sweeps run on the device (``hs_richardson_*``): the
residual is one fused SpMV kernel that also applies the previous correction,
the correction is the L1GS apply.  Vectors are CUDA tensors in the matrix
precision.  The reference's setup rule ``partsize = max(1, n ÷ nthreads)``
(:20) sizes partitions for CPU threads; a GPU builder takes its partsize from
the ``partsize`` argument or the builder's default.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import (ChebyshevFirst, ChebyshevFourth, DeviceSparseMatrix, L1GSPrecBuilder, SymmetricSweep, CPU,
               _ChebSmoother, _dev_ptr, _stream_ptr, _torch_dtype, build_smoother, smooth_ as _cheb_smooth)
from . import _lib as _L
from ._lib import check, lib

SWEEPS = 2   # Richardson sweeps per smooth! call (:27)


class HybridSmoother:
    """HybridSmoother{A, s, residual, correction} (:8-13) on the device."""

    def __init__(self, A, prec, stream=None):
        self.A = A if isinstance(A, DeviceSparseMatrix) else DeviceSparseMatrix(A)
        self.s = prec
        self._h = C.c_void_p()
        self._destroy = _L.lib().hs_richardson_destroy
        check(lib().hs_richardson_create(self.A.handle, prec.handle, C.byref(self._h)))

    def __del__(self):
        h = getattr(self, "_h", None)
        destroy = getattr(self, "_destroy", None)
        if h and destroy is not None:
            try:
                destroy(h)
            except Exception:
                pass
            self._h = None


def setup_smoother(config, A, symmetry=None, partsize=None, stream=None):
    """AMG.setup_smoother(config, A, symmetry) (:15-24, :35-41)."""
    if isinstance(config, L1GSPrecBuilder):
        if isinstance(config.backend, CPU):
            raise NotImplementedError("the KA.CPU() backend is not part of this library (B200 only)")
        prec = config(A, partsize, sweep=SymmetricSweep(), isSymA=False, stream=stream)   # :21
        return HybridSmoother(A, prec, stream)
    if isinstance(config, (ChebyshevFourth, ChebyshevFirst)):
        return build_smoother(config, A, stream)
    raise TypeError(f"no AMG smoother for {type(config).__name__}")


def smooth_(x, s, b, stream=None, sweeps=SWEEPS):
    """AMG.smooth!(x, s, b) (:26-33, :43-49): x updated in place."""
    if isinstance(s, _ChebSmoother):
        return _cheb_smooth(x, s, b, stream)
    td = _torch_dtype(_L.HS_F64 if s.A.dtype == np.float64 else _L.HS_F32)
    check(lib().hs_richardson_smooth(s._h, _dev_ptr(x, td), _dev_ptr(b, td), int(sweeps), _stream_ptr(stream)))
