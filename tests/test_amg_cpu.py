"""AMG smoother host logic without a GPU: configuration errors of
setup_smoother and the smoothing property of the oracle restatement."""
import numpy as np
import pytest

import hsb200
from hsb200 import amg
from hsb200 import workloads as W
from oracle import hs_oracle as O


def test_setup_smoother_rejects_cpu_and_unknown_configs():
    A = W.poisson_test_matrix(64)
    with pytest.raises(NotImplementedError):
        amg.setup_smoother(hsb200.L1GSPrecBuilder(hsb200.CPU(), chunks=4), A)
    with pytest.raises(TypeError):
        amg.setup_smoother(object(), A)


def test_oracle_richardson_smooths():
    A = W.poisson2d_matrix(30, eps=1.0)
    n = A.shape[0]
    xs = np.random.default_rng(4).uniform(-1, 1, n)
    b = A @ xs
    P = O.OracleL1GS(A, 16, isSymA=False, sweep="symmetric", cache="packed")
    x = np.zeros(n)
    prev = np.linalg.norm(b)
    for _ in range(3):
        x = O.amg_richardson(A, P, x, b)
        res = np.linalg.norm(b - A @ x)
        assert res < prev
        prev = res
