"""Serving and batching around the smoother path (no counterpart in the
reference, whose callers solve one system at a time through LinearSolve).

* ``BatchEngine`` wraps the C engine (``hs_batch_*``): each admitted system
  keeps its FP64 matrix, an FP32 L1GS SymmetricSweep packed preconditioner and
  its PCG state in HBM; one ``step`` advances every active system with a
  replayed CUDA graph of per-phase launches (or, ``schedule="persistent"``,
  one graph-captured persistent launch for all the step's iterations).  Admission is refused while no slot or not enough
  of the HBM budget is free.
* ``serve`` replays a timed request stream with continuous batching: requests
  that arrive while others are on the GPU are admitted as slots and memory free
  up, their setup overlaps the running iterations, and finished systems leave
  at the next step.  It reports solves/s and p50/p99 latency
  (arrival -> solution on the host).
* ``solve_sequential`` is the plain drop-in: one FP64 L1GS-preconditioned PCG
  solve after another, no batching.
"""
from __future__ import annotations

import ctypes as C
import time
from collections import deque

import numpy as np

from . import _lib as _L
from ._lib import check, lib


from ._lib import hs_batch_config, hs_batch_info, hs_batch_result  # noqa: E402


SCHEDULES = {"persistent": _L.HS_BATCH_PERSISTENT, "segmented": _L.HS_BATCH_SEGMENTED}


class BatchEngine:
    """schedule: "segmented" (a replayed CUDA graph of separate launches per
    iteration, each phase at its own occupancy; the faster) or "persistent"
    (one persistent kernel per launch runs all its iterations of all systems,
    work items from a device queue); the iterates are bitwise identical."""

    def __init__(self, max_slots=64, hbm_budget=64 << 30, partsize=16, rtol=1e-8, maxit=5000,
                 schedule="segmented"):
        import torch
        torch.cuda.init()
        if schedule not in SCHEDULES:
            raise ValueError(f"schedule must be one of {sorted(SCHEDULES)}")
        cfg = hs_batch_config(max_slots, int(hbm_budget), partsize, rtol, maxit, SCHEDULES[schedule])
        self._h = C.c_void_p()
        self._destroy = lib().hs_batch_destroy   # usable in __del__ at interpreter exit
        check(lib().hs_batch_create(C.byref(cfg), None, C.byref(self._h)))
        self._keep = {}      # tag -> (host sparse, b, x)

    def submit(self, A, b, tag, partsize=0):
        """Admit a system; returns False (nothing changed) when it does not fit now."""
        from . import _HostSparse
        hA = _HostSparse(A, dtype=np.float64)
        b = np.ascontiguousarray(b, dtype=np.float64)
        x = np.zeros_like(b)
        slot = C.c_int32()
        st = lib().hs_batch_submit(self._h, C.byref(hA.desc), b.ctypes.data_as(C.c_void_p),
                                   x.ctypes.data_as(C.c_void_p), int(tag), int(partsize), C.byref(slot))
        if st == _L.HS_ERR_BUDGET:
            return False
        check(st)
        self._keep[int(tag)] = (hA, b, x)
        return True

    def step(self, iters=4):
        nf = C.c_int32()
        check(lib().hs_batch_step(self._h, int(iters), C.byref(nf)))
        return nf.value

    def launch(self, iters=4):
        """Enqueue `iters` iterations of every active system and return at once."""
        check(lib().hs_batch_launch(self._h, int(iters)))

    def wait(self):
        """Block until the last launch is done; returns how many systems finished."""
        nf = C.c_int32()
        check(lib().hs_batch_wait(self._h, C.byref(nf)))
        return nf.value

    def poll(self):
        """[(tag, x, iterations, converged, relres)] of finished systems."""
        out = []
        buf = (hs_batch_result * 256)()
        while True:
            cnt = C.c_int32()
            check(lib().hs_batch_poll(self._h, buf, 256, C.byref(cnt)))
            for i in range(cnt.value):
                r = buf[i]
                _, _, x = self._keep.pop(int(r.tag))
                out.append((int(r.tag), x, int(r.iterations), bool(r.converged), float(r.relres)))
            if cnt.value < 256:
                break
        return out

    def info(self):
        i = hs_batch_info()
        check(lib().hs_batch_info_get(self._h, C.byref(i)))
        return i

    def close(self):
        if self._h:
            self._destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def percentile(v, q):
    return float(np.percentile(np.asarray(v, dtype=np.float64), q)) if len(v) else float("nan")


def serve(requests, max_slots=64, hbm_budget=64 << 30, iters_per_step=4, rtol=1e-8, partsize_of=None,
          realtime=True, maxit=5000, admit_per_step=8, tuner=None, engine_factory=None):
    """Continuous-batching replay of [(arrival_s, A, b)].

    partsize_of(A) -> 8/16/32 (e.g. Autotuner.partsize_of); default 16.
    tuner: an OnlineTuner (partsize_for(A, tag) at admission, observe(tag,
    iterations) when the solve finishes), which learns the partsize from
    the served solves themselves.  engine_factory(max_slots, hbm_budget,
    rtol, maxit) builds the engine (default: BatchEngine).  At most
    `admit_per_step` requests are admitted per step once systems are running,
    so their host-side preparation overlaps the GPU's iterations instead of
    delaying the first launch.
    Returns dict with per-request latency, iterations, results and totals.
    """
    factory = engine_factory or (lambda ms, hb, rt, mi: BatchEngine(max_slots=ms, hbm_budget=hb, rtol=rt, maxit=mi))
    eng = factory(max_slots, hbm_budget, rtol, maxit)
    order = sorted(range(len(requests)), key=lambda i: requests[i][0])
    pending = deque(order)
    waiting = deque()
    arrival = {}
    done_at, iters, conv, xs = {}, {}, {}, {}
    t0 = time.perf_counter()
    active = 0

    def admit():
        nonlocal active
        now = time.perf_counter() - t0
        while pending and (not realtime or requests[pending[0]][0] <= now):
            i = pending.popleft()
            arrival[i] = requests[i][0] if realtime else now
            waiting.append(i)
        admitted = 0
        while waiting and admitted < admit_per_step:
            i = waiting[0]
            _, A, b = requests[i]
            if tuner is not None:
                ps = tuner.partsize_for(A, i)
            else:
                ps = partsize_of(A) if partsize_of else 16
            if not eng.submit(A, b, i, ps):
                if tuner is not None:
                    tuner.cancel(i)   # not admitted now: its partsize is handed out again later
                break
            waiting.popleft()
            active += 1
            admitted += 1

    while pending or waiting or active:
        if active:
            # the GPU iterates while the host admits what has arrived meanwhile
            eng.launch(iters_per_step)
            admit()
            eng.wait()
            for tag, x, it, ok, rel in eng.poll():
                done_at[tag] = time.perf_counter() - t0
                iters[tag], conv[tag], xs[tag] = it, ok, x
                active -= 1
                if tuner is not None and tag in tuner.tags:
                    tuner.observe(tag, it)
        else:
            admit()
            if not active and waiting:
                # nothing runs, so nothing will free up: the head request can never fit
                raise RuntimeError(f"request {waiting[0]} cannot be admitted by an idle engine "
                                   f"(max_slots={max_slots}, hbm_budget={hbm_budget})")
            if not active and pending:
                wait = requests[pending[0]][0] - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
    total = time.perf_counter() - t0
    eng.close()
    lat = [done_at[i] - arrival[i] for i in done_at]
    return {"latency_s": lat, "iterations": iters, "converged": conv, "x": xs, "wall_s": total,
            "solves_per_s": len(done_at) / total, "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99)}


def solve_sequential(requests, partsize=16, rtol=1e-8, precision=None, maxit=5000):
    """The plain FP64 drop-in: build + PCG per request, one after the other."""
    import torch
    import hsb200
    t0 = time.perf_counter()
    lat, iters = [], []
    for arr, A, b in sorted(requests, key=lambda r: r[0]):
        ts = time.perf_counter()
        P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(
            A, partsize, isSymA=True, sweep=hsb200.SymmetricSweep(), cache_strategy=hsb200.PackedBufferCache(),
            precision=precision)
        M = hsb200.DeviceSparseMatrix(A)
        bd = torch.from_numpy(np.ascontiguousarray(b)).cuda()
        x = torch.zeros_like(bd)
        info = hsb200.pcg(M, bd, x, P, rtol=rtol, maxit=maxit)
        x.cpu()
        lat.append(time.perf_counter() - ts)
        iters.append(info.iterations)
        del P, M
    total = time.perf_counter() - t0
    return {"wall_s": total, "solves_per_s": len(requests) / total, "latency_s": lat, "iterations": iters,
            "p50_s": percentile(lat, 50), "p99_s": percentile(lat, 99)}


def serve_sharded(requests, **kw):
    """serve() across the ranks of a process group, one GPU each: rank r
    takes requests r, r + world, ... (each arrives at its own time) and runs
    its own engine; no collective touches the solves.  Returns, on every
    rank, the whole job's figures: solves/s = all solves / the slowest
    rank's wall time, p50/p99 over all requests, and {request: x}."""
    import torch.distributed as dist
    from . import distributed as D
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist.is_initialized() else (0, 1)
    mine = D.shard(list(range(len(requests))), rank, world)
    res = serve([requests[i] for i in mine], **kw)
    local = {"lat": res["latency_s"], "wall": res["wall_s"],
             "x": {mine[k]: v for k, v in res["x"].items()},
             "it": {mine[k]: v for k, v in res["iterations"].items()}}
    parts = [local]
    if world > 1:
        parts = [None] * world
        dist.all_gather_object(parts, local)
    lat = [t for p_ in parts for t in p_["lat"]]
    wall = max(p_["wall"] for p_ in parts)
    xs = {k: v for p_ in parts for k, v in p_["x"].items()}
    its = {k: v for p_ in parts for k, v in p_["it"].items()}
    return {"solves": len(xs), "wall_s": wall, "solves_per_s": len(xs) / wall, "p50_s": percentile(lat, 50),
            "p99_s": percentile(lat, 99), "x": xs, "iterations": its, "ranks": world}
