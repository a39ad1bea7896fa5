#!/usr/bin/env python
"""Benchmark of the HybridSmoothers.jl smoother-apply hot path on B200.

Headline workload: the 128^3 7-point Poisson operator (N = 2,097,152,
nnz = 14,581,760, FP64), L1 Gauss-Seidel SymmetricSweep with PackedBufferCache
at partsize 16 — one `ldiv!(y, P, x)` per step.  Metric: smoother GB/s on the
algorithmic bytes of one apply (8*(2S + 3N) for a fused symmetric packed sweep:
both packed triangles, D_Dl1, x read and y written once), and its fraction of
the measured HBM peak.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (under torchrun): every rank runs its own copy of the workload (the
partitions are independent; no collective on the data path) -> weak scaling,
value = total bytes of all ranks / max-over-ranks time.
`--impl reference` times the CPU restatement of the reference algorithm (the
reference is Julia and cannot run here) with all host threads, on rank 0.
"""
import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "hybridsmoothers.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

L2_BYTES = 126 * 1024 * 1024


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="poisson128-l1gs-sym-packed-ps16")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--soak-s", type=float, default=1.0, help="untimed load before timing, for clock samples")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# Workloads and algorithmic bytes
# ---------------------------------------------------------------------------
def parse_workload(name):
    # poisson128-l1gs-<sweep>-<cache>-ps<k>[-fp32]
    parts = name.split("-")
    if parts[0] != "poisson128" or parts[1] != "l1gs":
        raise SystemExit(f"unknown workload {name}")
    sweep = {"fwd": "forward", "bwd": "backward", "sym": "symmetric"}[parts[2]]
    cache = parts[3]
    ps = int(parts[4][2:])
    fp32 = len(parts) > 5 and parts[5] == "fp32"
    return dict(grid=128, sweep=sweep, cache=cache, ps=ps, fp32=fp32)


def packed_len(n, ps):
    nparts = -(-n // ps)
    lps = n - (nparts - 1) * ps
    return ps * (ps - 1) * (nparts - 1) // 2 + lps * (lps - 1) // 2


def algorithmic_bytes(n, nnz, ps, sweep, cache, tv, nonsym=False):
    """Per-apply bytes: packed Tv*(S + 3N) per direction, symmetric fused
    Tv*(2S + 3N); view nnz*(Ti+Tv) + (N+1)*Ti + 3*Tv*N (+ N*Ti for the
    non-symmetric DiagonalIndices path)."""
    ti = 4
    if cache == "packed":
        S = packed_len(n, ps)
        return tv * ((2 if sweep == "symmetric" else 1) * S + 3 * n)
    b = nnz * (ti + tv) + (n + 1) * ti + 3 * tv * n
    return b + (n * ti if nonsym else 0)


# ---------------------------------------------------------------------------
# Clock sampling (NVML) over the soak + timed window
# ---------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, dev_index, period_s=0.02):
        self.samples = []
        self.period = period_s
        self.dev_index = dev_index
        self._stop = threading.Event()
        self._t = None
        self.ok = False
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(dev_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((mhz, reasons))
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        if self.ok:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()

    def stop(self):
        if self._t:
            self._stop.set()
            self._t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unavailable"], "samples": 0}
        nv = self.nv
        names = {
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80),
        }
        seen = set()
        for _, r in self.samples:
            for k, bit in names.items():
                if r & bit:
                    seen.add(k)
        return {"sm_mhz": statistics.median(m for m, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(seen), "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# Measured peak (roofline denominator)
# ---------------------------------------------------------------------------
def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(workload):
    """dram bytes per launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        return json.load(open(p)).get(workload)
    except Exception:
        return None


# ---------------------------------------------------------------------------
# CPU leg (the oracle restatement; the reference itself is Julia)
# ---------------------------------------------------------------------------
def cpu_apply_rate(A, wl, x, budget_s=10.0, max_reps=None):
    from oracle import hs_oracle as O
    threads = O.omp_threads()
    dtype = np.float32 if wl["fp32"] else np.float64
    P = O.OracleL1GS(A, wl["ps"], isSymA=True, sweep=wl["sweep"], cache=wl["cache"], nchunks=threads,
                     chunksize=-(-(-(-A.shape[0] // wl["ps"])) // threads), dtype=dtype)
    xx = x.astype(dtype)
    y = np.empty_like(xx)
    P.ldiv(xx, out=y)  # warm
    reps, t0 = 0, time.perf_counter()
    while True:
        P.ldiv(xx, out=y)
        reps += 1
        el = time.perf_counter() - t0
        if el >= budget_s or (max_reps and reps >= max_reps):
            break
    return reps, el, threads


def main():
    args = parse_args()
    wl = parse_workload(args.workload)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    from hsb200 import workloads as W
    A = W.poisson3d_7pt(wl["grid"])
    n, nnz = A.shape[0], A.nnz
    x = W.rhs_uniform(n)
    tv = 4 if wl["fp32"] else 8
    bytes_per = algorithmic_bytes(n, nnz, wl["ps"], wl["sweep"], wl["cache"], tv)
    config = {"workload": args.workload, "grid": "128^3", "n": n, "nnz": nnz, "partsize": wl["ps"],
              "sweep": wl["sweep"], "cache": wl["cache"], "matrix": "7-point Poisson, Dirichlet, FP64 CSC",
              "parallelism": f"replicas{world}" if world > 1 else "single",
              "l2": f"inputs larger than L2 ({bytes_per / 2**20:.0f} MiB per apply vs 126 MiB L2)",
              "bytes_per_step": bytes_per}

    if args.impl == "reference":
        if rank != 0:
            return
        reps, el, threads = cpu_apply_rate(A, wl, x, budget_s=1e9, max_reps=args.warmup + args.steps)
        # time exactly `steps` applies after `warmup`
        from oracle import hs_oracle as O
        dtype = np.float32 if wl["fp32"] else np.float64
        P = O.OracleL1GS(A, wl["ps"], isSymA=True, sweep=wl["sweep"], cache=wl["cache"], nchunks=threads,
                         chunksize=-(-(-(-n // wl["ps"])) // threads), dtype=dtype)
        xx = x.astype(dtype)
        y = np.empty_like(xx)
        for _ in range(args.warmup):
            P.ldiv(xx, out=y)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            P.ldiv(xx, out=y)
        el = time.perf_counter() - t0
        v = bytes_per * args.steps / el / 1e9
        out = {"impl": "reference", "metric": "smoother GB/s (% HBM peak)", "value": round(v, 3), "unit": "GB/s",
               "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": round(el / args.steps * 1e3, 4), "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32" if wl["fp32"] else "f64", "data": "synthetic",
               "config": config,
               "cpu_baseline": {"value": round(v, 3), "unit": "GB/s", "cores": threads, "kind": "port",
                                "sample": f"{args.steps} full applies of the 128^3 workload (C restatement of "
                                          "the reference algorithm, OpenMP; the Julia reference cannot run here)"},
               "e2e": {"value": round(v, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return

    import torch
    import torch.distributed as dist
    import hsb200
    from hsb200 import _lib

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    stream = torch.cuda.current_stream()

    sweep = {"forward": hsb200.ForwardSweep(), "backward": hsb200.BackwardSweep(),
             "symmetric": hsb200.SymmetricSweep()}[wl["sweep"]]
    cache = hsb200.PackedBufferCache() if wl["cache"] == "packed" else hsb200.MatrixViewCache()
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(local_rank), threads=256, blocks=148)(
        A, wl["ps"], isSymA=True, sweep=sweep, cache_strategy=cache,
        precision=np.float32 if wl["fp32"] else None)
    tdt = torch.float32 if wl["fp32"] else torch.float64
    xd = torch.from_numpy(x).to(device="cuda", dtype=tdt)
    yd = torch.empty_like(xd)

    for _ in range(args.warmup):
        P.apply(xd, yd)
    torch.cuda.synchronize()

    clocks = ClockSampler(local_rank)
    clocks.start()
    # untimed soak so the clock record covers a loaded GPU
    t_end = time.perf_counter() + args.soak_s
    while time.perf_counter() < t_end:
        for _ in range(50):
            P.apply(xd, yd)
        torch.cuda.synchronize()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = hsb200.kernel_launches()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        P.apply(xd, yd)
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = hsb200.kernel_launches() - launches0
    ms = ev0.elapsed_time(ev1)
    clocks.stop()
    if world > 1:
        t = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()

    ms_step = ms / args.steps
    value = world * bytes_per * args.steps / (ms / 1e3) / 1e9
    kernel_gbs = bytes_per / (ms_step / 1e3) / 1e9
    peak, peak_src = hbm_peak()

    # e2e: the same apply through the C ABI with pinned host vectors
    e2e = None
    if not args.no_e2e:
        xh = torch.empty(n, dtype=tdt, pin_memory=True)
        xh.copy_(torch.from_numpy(x).to(tdt))
        yh = torch.empty(n, dtype=tdt, pin_memory=True)
        io = _lib.HS_F32 if wl["fp32"] else _lib.HS_F64
        import ctypes
        sp_ = ctypes.c_void_p(stream.cuda_stream)

        def host_step():
            _lib.check(hsb200.lib().hs_l1gs_apply_host(P.handle, ctypes.c_void_p(xh.data_ptr()),
                                                      ctypes.c_void_p(yh.data_ptr()), io, sp_))
        for _ in range(args.warmup):
            host_step()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            host_step()
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ems], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e = {"value": round(world * bytes_per * args.steps / (ems / 1e3) / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": n * tv, "d2h_bytes_per_step": n * tv,
               "ms_per_step": round(ems / args.steps, 4)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        reps, el, threads = cpu_apply_rate(A, wl, x, budget_s=10.0)
        cpu = {"value": round(bytes_per * reps / el / 1e9, 3), "unit": "GB/s", "cores": threads, "kind": "port",
               "sample": f"{reps} full applies of the 128^3 workload in {el:.1f} s (C restatement of the "
                         "reference algorithm, OpenMP over partitions)"}

    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    out = {
        "metric": "smoother GB/s (% HBM peak)", "value": round(value, 3), "unit": "GB/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms_step, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32" if wl["fp32"] else "f64", "data": "synthetic",
        "config": config,
        "roofline": {"bound": "hbm", "achieved": round(kernel_gbs, 2), "peak": peak, "unit": "GB/s",
                     "frac": round(kernel_gbs / peak, 4), "peak_source": peak_src,
                     "traffic": profiled_traffic(args.workload)},
        "hbm_frac_of_measured": round(kernel_gbs / peak, 4),
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
    }
    print(json.dumps(out))


if __name__ == "__main__":
    main()
