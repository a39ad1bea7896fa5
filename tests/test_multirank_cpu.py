"""The N>1 path on CPU: two gloo ranks exercise the host logic the multi-GPU
bench uses (round-robin sharding of work, max-over-ranks timing, sum of
processed units) and a shard solved by each rank with the oracle matches the
single-process answer."""
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
