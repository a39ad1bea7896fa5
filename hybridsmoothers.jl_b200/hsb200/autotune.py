"""Per-matrix choice of the L1GS partsize (and packed vs view storage) for the
served/batched PCG.

The cost of a solve is (iterations to 1e-8) x (time per iteration); partsize
trades the first against the second (a larger block captures more coupling but
streams ps/2 more values per row and sweep).  The tuner measures, for each
candidate, a short PCG run on the actual matrix: the residual reduction per
second over `trial_iters` iterations.  Decisions are cached per matrix class
(stencil width and size bucket), so a stream of similar requests pays the
trial once per class.
"""
from __future__ import annotations

import math
import time

import numpy as np

CANDIDATES = (8, 16, 32)


def matrix_class(A):
    n = A.shape[0]
    width = int(round(A.nnz / max(n, 1)))
    return (width, int(round(math.log2(max(n, 2)))))


class Autotuner:
    def __init__(self, candidates=CANDIDATES, trial_iters=30, precision=np.float32, caches=("packed",)):
        self.candidates = tuple(candidates)
        self.trial_iters = trial_iters
        self.precision = precision
        self.caches = tuple(caches)
        self.cache = {}
        self.trials = []

    def rate(self, A, ps, cache="packed"):
        """log10 residual reduction per second of a short PCG run with partsize ps."""
        import torch
        import hsb200
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, ps, isSymA=True, sweep=hsb200.SymmetricSweep(),
            cache_strategy=hsb200.PackedBufferCache() if cache == "packed" else hsb200.MatrixViewCache(),
            precision=self.precision)
        M = hsb200.DeviceSparseMatrix(A)
        b = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, A.shape[0])).cuda()
        x = torch.zeros_like(b)
        info = hsb200.pcg(M, b, x, P, rtol=1e-30, maxit=self.trial_iters)   # fixed-length run
        rel = max(info.relres, 1e-300)
        secs = max(info.ms * 1e-3, 1e-9)
        return -math.log10(rel) / secs

    def choose(self, A):
        key = matrix_class(A)
        if key in self.cache:
            return self.cache[key]
        best, best_rate = None, -1.0
        t0 = time.perf_counter()
        for cache in self.caches:
            for ps in self.candidates:
                r = self.rate(A, ps, cache)
                if r > best_rate:
                    best, best_rate = (ps, cache), r
        self.trials.append((key, best, time.perf_counter() - t0))
        self.cache[key] = best
        return best

    def partsize_of(self, A):
        return self.choose(A)[0]
