"""The N>1 path on CPU: two gloo ranks exercise the host logic the multi-GPU
bench uses (round-robin sharding of work, max-over-ranks timing, sum of
processed units) and a shard solved by each rank with the oracle matches the
single-process answer; serve_sharded (the served stream split across ranks,
one engine per rank) runs with an engine double whose solves are the
oracle's, and gathers every request exactly once."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "hybridsmoothers.jl_b200")]
    import torch.distributed as dist
    from hsb200 import distributed as D
    from hsb200 import workloads as W
    from oracle import hs_oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = W.serving_stream(count=6, lo=200, hi=900, seed=9)
        mine = D.shard(list(range(len(reqs))), rank, world)
        sols = {}
        for i in mine:
            _, A, b = reqs[i]
            x, it, rel = O.pcg(A, b, O.OracleL1GS(A, 8, isSymA=True, sweep="symmetric", cache="packed"))
            assert it > 0 and rel < 1e-7
            sols[i] = x
        t = D.max_over_ranks(0.5 + rank)          # rank-dependent fake timing
        units = D.sum_over_ranks(len(mine))
        gathered = [None] * world
        dist.all_gather_object(gathered, sols)
        q.put((rank, t, units, {k: v.tolist() for g in gathered for k, v in g.items()}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from hsb200 import workloads as W
    from oracle import hs_oracle as O
    reqs = W.serving_stream(count=6, lo=200, hi=900, seed=9)
    for rank, t, units, sols in out:
        assert t == 1.5                      # max over ranks
        assert units == len(reqs)            # every request processed exactly once
        assert sorted(sols) == list(range(len(reqs)))
        for i, xs in sols.items():
            _, A, b = reqs[int(i)]
            x, _, _ = O.pcg(A, b, O.OracleL1GS(A, 8, isSymA=True, sweep="symmetric", cache="packed"))
            np.testing.assert_array_equal(np.array(xs), x)


def test_shard_partition():
    from hsb200 import distributed as D
    items = list(range(11))
    parts = [D.shard(items, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == items
    assert all(len(p) in (3, 4) for p in parts)


class OracleEngine:
    """Stands in for BatchEngine on CPU: submit solves with the oracle's PCG,
    poll hands the results back (the engine's interface, no GPU)."""

    def __init__(self, *args):
        self.done = []

    def submit(self, A, b, tag, partsize=0):
        from oracle import hs_oracle as O
        x, it, _ = O.pcg(A, b, O.OracleL1GS(A, partsize or 8, isSymA=True, sweep="symmetric", cache="packed"))
        self.done.append((int(tag), x, it, it > 0, 0.0))
        return True

    def launch(self, iters=4):
        pass

    def wait(self):
        return len(self.done)

    def poll(self):
        out, self.done = self.done, []
        return out

    def close(self):
        pass


def _serve_worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "hybridsmoothers.jl_b200")]
    import torch.distributed as dist
    from hsb200 import serving
    from hsb200 import workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        reqs = W.serving_stream(count=7, lo=200, hi=900, seed=4)
        res = serving.serve_sharded([(0.0, A, b) for _, A, b in reqs], realtime=False,
                                    partsize_of=lambda A: 8, engine_factory=lambda *a: OracleEngine())
        q.put((rank, res["solves"], res["ranks"], {k: v.tolist() for k, v in res["x"].items()}))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_serve_sharded():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_serve_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    from hsb200 import workloads as W
    from oracle import hs_oracle as O
    reqs = W.serving_stream(count=7, lo=200, hi=900, seed=4)
    for rank, solves, ranks, xs in out:
        assert solves == len(reqs) and ranks == 2
        assert sorted(xs) == list(range(len(reqs)))
        for i, x in xs.items():
            _, A, b = reqs[int(i)]
            xr, _, _ = O.pcg(A, b, O.OracleL1GS(A, 8, isSymA=True, sweep="symmetric", cache="packed"))
            np.testing.assert_array_equal(np.array(x), xr)
