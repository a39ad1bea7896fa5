"""The ordering protocol of the batched engine's persistent launch
(hs_batch_config.schedule = HS_BATCH_PERSISTENT, csrc/batch.cu
batch_persistent_kernel), modelled on the CPU.

A launch's work items are ordered by (iteration, phase, slot, chunk); CTAs take
kTake consecutive items per ticket and run them in order.  A slot's first item
of a phase (its closer) waits until the slot's previous phase is open (its
stage) and all of its items are counted, then publishes the slot's stage; the
phase's other items wait for the stage.  A slot that converges at a check (closer of phase 2) is marked finished
and its remaining items are skipped.

The model runs that protocol with every CTA a separate actor, interleaved at
random, and checks: the launch always finishes (no deadlock) for any number of
resident CTAs, including one; no item runs before every item of its slot's
previous phase has finished; and finished slots run nothing more.
"""
import random

import pytest

K_TAKE = 4
DONE = 1 << 30


def work_table(slots):
    """slots: list of (chunks, groups) -> items of one iteration as
    (slot, phase, closer, count) in the kernel's order (2 chunks or 16 groups per item)."""
    table = []
    for ph in range(4):
        for s, (nblk, ngroups) in enumerate(slots):
            if ph == 2:
                for g in range(0, ngroups, 16):
                    table.append((s, 2, g == 0, min(16, ngroups - g)))
            else:
                for b in range(0, nblk, 2):
                    table.append((s, ph, b == 0, min(2, nblk - b)))
    return table


def phase_items(slot, ph):
    nblk, ngroups = slot
    return (ngroups + 15) // 16 if ph == 2 else (nblk + 1) // 2


def run_launch(slots, iters, ctas, converge_at, rng, closer_checks_stage=True):
    """converge_at[s]: iteration whose check ends slot s (None: never).
    closer_checks_stage=False drops the closer's stage condition (a planted
    mistake: the counter may still hold the phase before the previous one)."""
    table = work_table(slots)
    total = len(table) * iters
    stage = [0] * len(slots)
    fin = [0] * len(slots)
    ticket = [0]
    finished_items = {}     # (t, slot, phase) -> items finished
    ran = []
    # per CTA: None (idle) or [list of item indices, position, state]
    cta = [None] * ctas
    steps = 0
    live = set(range(ctas))
    while live:
        steps += 1
        assert steps < 200 * (total + ctas) + 1000, "no progress: deadlock"
        c = rng.choice(sorted(live))
        st = cta[c]
        if st is None:
            w0 = ticket[0] * K_TAKE
            ticket[0] += 1
            if w0 >= total:
                live.discard(c)
                continue
            cta[c] = [list(range(w0, min(total, w0 + K_TAKE))), 0]
            continue
        wi = st[0][st[1]]
        t, k = divmod(wi, len(table))
        s, ph, closer, count = table[k]
        need = 4 * t + ph
        closing = closer and not (t == 0 and ph == 0)
        if stage[s] >= DONE:
            go = "skip"
        elif closing:
            # the previous phase must be the one being counted (opened: stage
            # need - 1) and all of it counted
            ok = (stage[s] >= need - 1 or not closer_checks_stage) and \
                fin[s] >= phase_items(slots[s], (ph + 3) % 4)
            go = "run" if ok else "wait"
        else:
            go = "run" if stage[s] >= need else "wait"
        if go == "wait":
            continue            # poll again later
        if go == "run":
            # the dependency this protocol promises
            prev_t, prev_ph = (t, ph - 1) if ph > 0 else (t - 1, 3)
            if prev_t >= 0:
                assert finished_items.get((prev_t, s, prev_ph), 0) == phase_items(slots[s], prev_ph)
            if closing:
                fin[s] = 0
                stage[s] = need
                if ph == 2 and converge_at[s] == t:
                    stage[s] = DONE
                    go = "skip"
            if go == "run":
                ran.append((t, s, ph))
                fin[s] += 1
                key = (t, s, ph)
                finished_items[key] = finished_items.get(key, 0) + 1
        st[1] += 1
        if st[1] == len(st[0]):
            cta[c] = None
    return ran, stage


@pytest.mark.parametrize("seed", range(12))
def test_persistent_protocol_finishes_and_orders(seed):
    rng = random.Random(seed)
    nslots = rng.randint(1, 6)
    slots = [(rng.randint(1, 9), rng.randint(1, 40)) for _ in range(nslots)]
    iters = rng.randint(1, 4)
    ctas = rng.choice([1, 2, 3, 7, 16])
    converge_at = [rng.choice([None, None, rng.randrange(iters)]) for _ in range(nslots)]
    ran, stage = run_launch(slots, iters, ctas, converge_at, rng)
    for s in range(nslots):
        phases = [(t, ph) for (t, ss, ph) in ran if ss == s]
        # nothing after the check that finished the slot
        if converge_at[s] is not None:
            ct = converge_at[s]
            assert all((t, ph) <= (ct, 1) for t, ph in phases)
            assert stage[s] == DONE
        else:
            counts = {}
            for t, ph in phases:
                counts[(t, ph)] = counts.get((t, ph), 0) + 1
            for t in range(iters):
                for ph in range(4):
                    assert counts[(t, ph)] == phase_items(slots[s], ph)


def test_single_cta_runs_everything_in_order():
    rng = random.Random(5)
    slots = [(3, 20), (1, 1), (5, 33)]
    ran, _ = run_launch(slots, 2, 1, [None, None, None], rng)
    keys = [(t, ph, s) for (t, s, ph) in ran]
    assert keys == sorted(keys)


def test_model_catches_a_closer_without_the_stage_check():
    """With the closer's stage condition removed, a closer can see the counter
    of the phase before its previous one and open its phase early; the model's
    dependency check must catch that on some interleaving."""
    caught = 0
    for seed in range(40):
        rng = random.Random(seed)
        slots = [(rng.randint(3, 9), rng.randint(1, 20)) for _ in range(rng.randint(1, 4))]
        try:
            run_launch(slots, 2, 7, [None] * len(slots), rng, closer_checks_stage=False)
        except AssertionError:
            caught += 1
    assert caught > 0
