"""Per-matrix choice of the L1GS configuration: partsize, packed vs view
storage, and threads per partition (one thread per partition, or lanes of a
warp sharing one).  No counterpart in the reference, whose partsize and
cache_strategy are the caller's arguments (src/l1_gauss_seidel.jl:287-296,
:613-614).

The cost of a solve is (iterations to the tolerance) x (time per iteration).
Partsize moves both: a larger block captures more coupling (fewer iterations)
but streams more values per row.  Storage and threads per partition change
only the time per iteration (the preconditioner is the same operator).  So
the tuner measures, per matrix class:

1. for every candidate partsize, the residual reduction per iteration of a
   short fixed-length PCG run (the convergence rate);
2. for every (partsize, cache, threads per partition) candidate, the device
   time of one PCG iteration: the apply timed with CUDA events plus the SpMV
   and vector work, measured once;

and picks the candidate with the highest reduction per second.  Decisions are
cached per matrix class (stencil width and size bucket) together with the
trial cost.

``OnlineTuner`` serves the batched engine, which offers partsizes 8/16/32 of
the packed FP32 smoother: it spends no trial work, but gives small requests
of a class the candidates in turn and, once each has finished, keeps the one
with the fewest modelled bytes to convergence (iterations x bytes streamed
per iteration; the batched kernels are bandwidth-bound).  Classes are coarse
(stencil width buckets), and iteration counts are compared per n^(1/d) (d = 2
for widths up to 5, else 3: PCG iterations of a stencil operator grow like
h^-1), so requests of different sizes inform one choice; large requests never
explore.
"""
from __future__ import annotations

import math
import time

import numpy as np

PARTSIZES = (8, 12, 16, 24, 32, 64, 128, 256)
CACHES = ("packed", "view")
THREADS = (1, 0)   # one thread per partition, or the library's lanes-per-partition choice


def matrix_class(A):
    n = A.shape[0]
    width = int(round(A.nnz / max(n, 1)))
    return (width, int(round(math.log2(max(n, 2)))))


def _build(A, ps, cache, tpp, precision):
    import hsb200
    order = "reference" if tpp == 1 else "any"
    return hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
        A, ps, isSymA=True, sweep=hsb200.SymmetricSweep(),
        cache_strategy=hsb200.PackedBufferCache() if cache == "packed" else hsb200.MatrixViewCache(),
        precision=precision, threads_per_part=tpp if tpp == 1 else 0, order=order)


def _time_apply(P, n, reps=5):
    import torch
    import hsb200
    x = torch.ones(n, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    hsb200.ldiv_(y, P, x)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        hsb200.ldiv_(y, P, x)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


class Autotuner:
    def __init__(self, partsizes=PARTSIZES, caches=CACHES, threads=THREADS, trial_iters=20, precision=None):
        self.partsizes = tuple(partsizes)
        self.caches = tuple(caches)
        self.threads = tuple(threads)
        self.trial_iters = trial_iters
        self.precision = precision
        self.cache = {}     # class -> (ps, cache, threads_per_part)
        self.trials = []    # (class, choice, trial seconds, {candidate: score})

    def _rate(self, A, M, b, ps):
        """log10 residual reduction per iteration of a fixed-length PCG run,
        and the device time of one iteration without the preconditioner."""
        import torch
        import hsb200
        P = _build(A, ps, "packed", 0, self.precision)
        x = torch.zeros_like(b)
        info = hsb200.pcg(M, b, x, P, rtol=1e-30, maxit=self.trial_iters)
        rel = max(info.relres, 1e-300)
        return -math.log10(rel) / max(info.iterations, 1)

    def choose(self, A):
        """(partsize, cache, threads_per_part) for A; threads_per_part 0 means
        the library's lanes-per-partition choice."""
        import torch
        import hsb200
        key = matrix_class(A)
        if key in self.cache:
            return self.cache[key]
        t0 = time.perf_counter()
        n = A.shape[0]
        M = hsb200.DeviceSparseMatrix(A)
        b = torch.from_numpy(np.random.default_rng(0).uniform(-1, 1, n)).cuda()
        # the iteration's work besides the preconditioner: one unpreconditioned PCG iteration
        x = torch.zeros_like(b)
        hsb200.pcg(M, b, x, None, rtol=1e-30, maxit=2)
        base = hsb200.pcg(M, b, x, None, rtol=1e-30, maxit=self.trial_iters)
        t_base = base.ms * 1e-3 / max(base.iterations, 1)
        scores = {}
        for ps in self.partsizes:
            if ps >= n:
                continue
            rate = self._rate(A, M, b, ps)
            for cache in self.caches:
                for tpp in self.threads:
                    try:
                        P = _build(A, ps, cache, tpp, self.precision)
                    except (NotImplementedError, ValueError):
                        continue
                    if tpp == 0 and P.threads_per_part == 1:
                        continue   # the library keeps one thread per partition here: same as tpp 1
                    t_apply = _time_apply(P, n)
                    scores[(ps, cache, P.threads_per_part if tpp == 0 else 1)] = rate / (t_base + t_apply)
                    del P
        best = max(scores, key=scores.get)
        choice = (best[0], best[1], best[2] if best[2] == 1 else 0)
        self.trials.append((key, choice, time.perf_counter() - t0, scores))
        self.cache[key] = choice
        return choice

    def build(self, A):
        """The chosen preconditioner for A."""
        ps, cache, tpp = self.choose(A)
        return _build(A, ps, cache, tpp, self.precision)

    def partsize_of(self, A):
        return self.choose(A)[0]


def batch_bytes_per_iteration(n, nnz, ps):
    """Bytes one batched PCG iteration streams for a system: the FP64 CSR
    SpMV, the FP32 symmetric packed sweep (both triangles, D_Dl1, y in/out),
    and the PCG vectors."""
    nparts = -(-n // ps)
    lps = n - (nparts - 1) * ps
    S = ps * (ps - 1) * (nparts - 1) // 2 + lps * (lps - 1) // 2
    return 12 * nnz + 4 * (n + 1) + 4 * (2 * S + 3 * n) + 8 * 12 * n


def serving_class(A):
    """(width bucket, dimension) of the online tuner: widths up to 5, 6-9,
    10-19, 20 and more."""
    width = A.nnz / max(A.shape[0], 1)
    bucket = 0 if width <= 5.5 else 1 if width <= 9.5 else 2 if width <= 19.5 else 3
    return (bucket, 2 if bucket == 0 else 3)


class OnlineTuner:
    """Partsize of the batched engine's FP32 smoother, learnt from the solves
    themselves: per class, each candidate is tried on a small request (n at
    most `explore_max_n`); the finished solves' iteration counts, scaled by
    n^(1/d), pick the partsize with the fewest modelled bytes to
    convergence.  Until then (and for large requests) the default runs."""

    def __init__(self, candidates=(8, 16, 32), default=8, explore_max_n=1 << 17):
        self.candidates = tuple(candidates)
        self.default = default
        self.explore_max_n = explore_max_n
        self.assigned = {}   # class -> candidates handed out for exploration so far
        self.obs = {}        # class -> {ps: [normalised bytes to convergence per row, ...]}
        self.tags = {}       # tag -> (class, ps, n, nnz, exploring)
        self.history = {}    # tag -> partsize it ran with (admitted requests)

    def partsize_for(self, A, tag):
        key = serving_class(A)
        n = A.shape[0]
        done = self.obs.get(key, {})
        tried = self.assigned.setdefault(key, [])
        untried = [c for c in self.candidates if c not in tried]
        exploring = False
        if all(c in done for c in self.candidates):
            ps = min(self.candidates, key=lambda c: float(np.mean(done[c])))
        elif untried and n <= self.explore_max_n:
            ps = untried[0]
            tried.append(ps)
            exploring = True
        else:
            ps = self.default   # candidates still running, or a large request: the default
        self.tags[tag] = (key, ps, n, A.nnz, exploring)
        self.history[tag] = ps
        return ps

    def cancel(self, tag):
        """The request `tag` was not admitted: forget its assignment."""
        key, ps, _, _, exploring = self.tags.pop(tag)
        self.history.pop(tag, None)
        tried = self.assigned.get(key, [])
        if exploring and ps in tried:
            tried.remove(ps)

    def observe(self, tag, iterations):
        key, ps, n, nnz, _ = self.tags.pop(tag)
        n = max(n, 1)
        cost = iterations / n ** (1.0 / key[1]) * batch_bytes_per_iteration(n, nnz, ps) / n
        self.obs.setdefault(key, {}).setdefault(ps, []).append(cost)
        if ps not in self.assigned.setdefault(key, []):
            self.assigned[key].append(ps)   # a default run counts as that candidate's trial

    def choice(self, A):
        key = serving_class(A)
        done = self.obs.get(key, {})
        if not done:
            return None
        return min(done, key=lambda c: float(np.mean(done[c])))
