"""Batched / served PCG (hs_batch_*): correctness, isolation and admission.

* Every batched solve reaches ||b - A x|| <= ~1e-8 ||b|| and matches the
  single-system device PCG with the same FP32 smoother within +-1 iteration.
* A system's result is the same alone and in a mix of other systems — the
  stated tolerance is exact equality (per-slot reductions use fixed blocks and
  a fixed-order finalize).
* Admission is refused beyond the HBM budget / slot count and succeeds once
  memory frees up.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import serving
from hsb200 import workloads as W

pytestmark = pytest.mark.gpu


def small_stream(count, seed, lo=800, hi=40000):
    return W.serving_stream(count=count, lo=lo, hi=hi, seed=seed)


def true_relres(A, x, b):
    return np.linalg.norm(b - A @ x) / np.linalg.norm(b)


def single_pcg_iters(A, b, ps):
    P = hsb200.L1GSPrecBuilder(hsb200.CUDABackend(), threads=256, blocks=148)(A, ps, isSymA=True,
                                                                             precision=np.float32,
                                                                             order="reference")
    M = hsb200.DeviceSparseMatrix(A)
    bd = torch.from_numpy(b).cuda()
    x = torch.zeros_like(bd)
    info = hsb200.pcg(M, bd, x, P, rtol=1e-8)
    return info.iterations


@pytest.mark.parametrize("ps", [8, 16, 32])
def test_batch_solves_match_single(ps):
    reqs = small_stream(6, seed=ps)
    eng = serving.BatchEngine(max_slots=16)
    for i, (_, A, b) in enumerate(reqs):
        assert eng.submit(A, b, i, ps)
    results = {}
    for _ in range(2000):
        eng.step(8)
        for tag, x, it, ok, rel in eng.poll():
            results[tag] = (x, it, ok, rel)
        if len(results) == len(reqs):
            break
    assert len(results) == len(reqs)
    for i, (_, A, b) in enumerate(reqs):
        x, it, ok, rel = results[i]
        assert ok and rel <= 1e-8
        assert true_relres(A, x, b) <= 5e-8
        assert abs(it - single_pcg_iters(A, b, ps)) <= 1
    eng.close()


@pytest.mark.parametrize("schedule", ["segmented", "persistent"])
def test_same_result_alone_and_in_mix(schedule):
    reqs = small_stream(8, seed=11)
    target = reqs[3]
    # alone
    eng = serving.BatchEngine(max_slots=8, schedule=schedule)
    eng.submit(target[1], target[2], 0, 16)
    alone = None
    while alone is None:
        eng.step(4)
        for tag, x, it, ok, rel in eng.poll():
            alone = (x.copy(), it)
    eng.close()
    # in a mix, admitted after others are already iterating
    eng = serving.BatchEngine(max_slots=8, schedule=schedule)
    for i in (0, 1, 2):
        eng.submit(reqs[i][1], reqs[i][2], 100 + i, (8, 16, 32)[i % 3])
    eng.step(3)
    eng.submit(target[1], target[2], 0, 16)
    for i in (4, 5):
        eng.submit(reqs[i][1], reqs[i][2], 100 + i, 32)
    mixed = None
    for _ in range(5000):
        eng.step(5)
        for tag, x, it, ok, rel in eng.poll():
            if tag == 0:
                mixed = (x.copy(), it)
        if mixed is not None:
            break
    eng.close()
    assert mixed is not None
    assert mixed[1] == alone[1]
    np.testing.assert_array_equal(mixed[0], alone[0])


def test_budget_admission():
    reqs = small_stream(4, seed=5, lo=20000, hi=30000)
    # each system's own budget figure, from an engine with room for it
    need = []
    for _, A, b in reqs:
        probe = serving.BatchEngine(max_slots=1, hbm_budget=1 << 30)
        assert probe.submit(A, b, 0, 16)
        need.append(probe.info().hbm_used)
        probe.close()
    budget = max(need)
    two = sorted(need)[:2]
    assert budget < two[0] + two[1]   # room for one of these systems at a time
    eng = serving.BatchEngine(max_slots=8, hbm_budget=budget)
    admitted = [eng.submit(A, b, i, 16) for i, (_, A, b) in enumerate(reqs)]
    assert admitted[0] and not all(admitted)
    done = set()
    for _ in range(5000):
        eng.step(8)
        for tag, *_ in eng.poll():
            done.add(tag)
        for i, ok in enumerate(admitted):
            if not ok and eng.submit(reqs[i][1], reqs[i][2], i, 16):
                admitted[i] = True
        if len(done) == len(reqs):
            break
    assert len(done) == len(reqs)
    info = eng.info()
    assert info.active == 0 and info.hbm_used == 0
    eng.close()


def test_serve_stream_reports_latency():
    reqs = small_stream(24, seed=3)
    # arrivals spread over 0.2 s
    rng = np.random.default_rng(0)
    t = np.cumsum(rng.exponential(0.2 / 24, size=24))
    reqs = [(float(t[i]), A, b) for i, (_, A, b) in enumerate(reqs)]
    out = serving.serve(reqs, max_slots=8, iters_per_step=4)
    assert len(out["latency_s"]) == 24 and all(out["converged"].values())
    assert out["p99_s"] >= out["p50_s"] > 0
    for i, (_, A, b) in enumerate(reqs):
        assert true_relres(A, out["x"][i], b) <= 5e-8


def test_autotuner_picks_a_candidate():
    from hsb200.autotune import Autotuner
    A = W.variable_diffusion((24, 24, 24), np.random.default_rng(1))
    tuner = Autotuner(partsizes=(8, 16, 32), trial_iters=10)
    ps, cache, tpp = tuner.choose(A)
    assert ps in (8, 16, 32) and cache in ("packed", "view") and tpp in (0, 1)
    assert tuner.choose(A) == (ps, cache, tpp)   # cached by matrix class


@pytest.mark.parametrize("schedule", ["segmented", "persistent"])
def test_admission_during_launch_reuses_slot(schedule):
    """A system submitted while a launch is in flight, into the slot a
    finished system just left, joins at the next launch: the in-flight copy
    of that slot's scalars (the previous occupant's, converged) must not mark
    it finished, and its result equals the alone result bitwise."""
    reqs = small_stream(2, seed=23)
    (_, A1, b1), (_, A2, b2) = reqs
    eng = serving.BatchEngine(max_slots=1, schedule=schedule)
    assert eng.submit(A1, b1, 1, 8)
    first = None
    while first is None:
        eng.step(8)
        for tag, x, it, ok, rel in eng.poll():
            first = (tag, it, ok)
    assert first[0] == 1 and first[2]
    eng.launch(4)                      # nothing active: only the scalars copy is in flight
    assert eng.submit(A2, b2, 2, 8)    # same slot, admitted during the launch
    assert eng.wait() == 0
    assert eng.poll() == []
    res = None
    for _ in range(2000):
        eng.launch(8)
        eng.wait()
        for tag, x, it, ok, rel in eng.poll():
            res = (tag, x.copy(), it, ok)
        if res:
            break
    eng.close()
    assert res is not None and res[0] == 2 and res[3]
    alone = serving.BatchEngine(max_slots=1, schedule=schedule)
    alone.submit(A2, b2, 0, 8)
    ref = None
    while ref is None:
        alone.step(8)
        for tag, x, it, ok, rel in alone.poll():
            ref = (x.copy(), it)
    alone.close()
    assert res[2] == ref[1]
    np.testing.assert_array_equal(res[1], ref[0])


def _finish_all(eng, count, iters, limit=3000):
    res = {}
    for _ in range(limit):
        eng.step(iters)
        for tag, x, it, ok, rel in eng.poll():
            res[tag] = (x.copy(), it, ok, rel)
        if len(res) == count:
            break
    return res


@pytest.mark.parametrize("maxit", [5000, 7])
def test_persistent_schedule_matches_segmented(maxit):
    """The persistent launch (one kernel per launch, work items from a device
    queue, each system's phases ordered by its own stage counter) and the
    segmented graph run the same arithmetic: solutions, iteration counts and
    flags are identical -- systems of all three partsizes, admitted in two
    waves, and (maxit 7) an iteration cap that stops every system."""
    reqs = small_stream(7, seed=31)
    out = {}
    for sched in ("persistent", "segmented"):
        eng = serving.BatchEngine(max_slots=8, maxit=maxit, schedule=sched)
        for i in range(4):
            assert eng.submit(reqs[i][1], reqs[i][2], i, (8, 16, 32)[i % 3])
        eng.step(3)
        for i in range(4, 7):
            assert eng.submit(reqs[i][1], reqs[i][2], i, (8, 16, 32)[i % 3])
        out[sched] = _finish_all(eng, len(reqs), 6)
        assert eng.info().active == 0
        eng.close()
    assert len(out["persistent"]) == len(reqs) == len(out["segmented"])
    for i in range(len(reqs)):
        xp, itp, okp, relp = out["persistent"][i]
        xs, its, oks, rels = out["segmented"][i]
        assert (itp, okp, relp) == (its, oks, rels)
        np.testing.assert_array_equal(xp, xs)
        if maxit == 7:
            assert itp == 7 and not okp
        else:
            assert okp and relp <= 1e-8


@pytest.mark.parametrize("schedule", ["persistent", "segmented"])
def test_zero_rhs_finishes_at_admission(schedule):
    """b = 0 is solved by x = 0 at admission (0 iterations) while another
    system iterates beside it."""
    (_, A, b), = small_stream(1, seed=2)
    eng = serving.BatchEngine(max_slots=2, schedule=schedule)
    assert eng.submit(A, np.zeros_like(b), 0, 8)
    assert eng.submit(A, b, 1, 16)
    res = _finish_all(eng, 2, 8)
    eng.close()
    x0, it0, ok0, rel0 = res[0]
    assert it0 == 0 and ok0 and not np.any(x0)
    assert res[1][2] and true_relres(A, res[1][0], b) <= 5e-8


def test_schedule_argument_checked():
    with pytest.raises(ValueError):
        serving.BatchEngine(max_slots=1, schedule="fused")
