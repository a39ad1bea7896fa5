"""The single-system autotuner (hsb200/autotune.py:Autotuner) on the GPU:
it searches partsize x packed/view x threads per partition, returns the
candidate with the best measured residual reduction per second, caches the
decision per matrix class, and its choice solves (PCG to 1e-8) about as fast
as the best of the candidates timed end to end."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import workloads as W
from hsb200.autotune import Autotuner, _build, matrix_class

pytestmark = pytest.mark.gpu


def solve_ms(A, b, P, reps=3):
    M = hsb200.DeviceSparseMatrix(A)
    bd = torch.from_numpy(b).cuda()
    x = torch.zeros_like(bd)
    hsb200.pcg(M, bd, x, P, rtol=1e-8)
    return min(hsb200.pcg(M, bd, x, P, rtol=1e-8).ms for _ in range(reps))


def test_autotuner_picks_a_fastest_candidate():
    A = W.poisson3d_7pt(64)
    b = W.rhs_uniform(A.shape[0])
    tuner = Autotuner(partsizes=(8, 16, 32, 64, 128), trial_iters=20)
    choice = tuner.choose(A)
    key, chosen, secs, scores = tuner.trials[-1]
    assert key == matrix_class(A) and chosen == choice and secs > 0
    assert {c[1] for c in scores} == {"packed", "view"}
    best = max(scores, key=scores.get)
    assert (best[0], best[1]) == (choice[0], choice[1])
    assert tuner.choose(A) is choice and len(tuner.trials) == 1   # cached per class
    # end to end: the choice against the worst-scored candidate and the default
    worst = min(scores, key=scores.get)
    t_choice = solve_ms(A, b, tuner.build(A))
    t_worst = solve_ms(A, b, _build(A, worst[0], worst[1], worst[2], None))
    t_default = solve_ms(A, b, _build(A, 16, "packed", 1, None))
    assert t_choice <= 1.25 * min(t_worst, t_default), (t_choice, t_worst, t_default)
