"""The serving tuner's decisions (hsb200/autotune.py:OnlineTuner), without a
GPU: candidates handed out in turn per matrix class, refused admissions
handed out again, and the partsize with the fewest modelled bytes to
convergence kept once every candidate has finished."""
import scipy.sparse as sp

from hsb200.autotune import OnlineTuner, batch_bytes_per_iteration, matrix_class
from hsb200 import workloads as W


def test_explores_then_exploits():
    A = W.poisson2d_matrix(40)
    B = W.poisson3d_7pt(12)
    assert matrix_class(A) != matrix_class(B)
    t = OnlineTuner(candidates=(8, 16, 32), default=16)
    got = [t.partsize_for(A, i) for i in range(3)]
    assert got == [8, 16, 32]
    assert t.partsize_for(A, 3) == 16          # nothing finished yet: the default
    assert t.partsize_for(B, 100) == 8         # another class explores on its own
    # 8 converges in fewer modelled bytes than 16 and 32
    n, nnz = A.shape[0], A.nnz
    iters = {0: 100, 1: 100, 2: 100}
    for tag, it in iters.items():
        t.observe(tag, it)
    t.observe(3, 100)
    costs = {ps: 100 * batch_bytes_per_iteration(n, nnz, ps) for ps in (8, 16, 32)}
    best = min(costs, key=costs.get)
    assert t.choice(A) == best
    assert t.partsize_for(A, 4) == best


def test_refused_admission_is_retried():
    A = W.poisson2d_matrix(30)
    t = OnlineTuner(candidates=(8, 16, 32))
    assert t.partsize_for(A, 0) == 8
    assert t.partsize_for(A, 1) == 16
    t.cancel(0)                                 # request 0 was not admitted
    assert t.partsize_for(A, 2) == 8            # 8 is handed out again
    assert t.partsize_for(A, 0) == 32


def test_bytes_model_grows_with_partsize():
    A = sp.identity(1000, format="csr")
    b = [batch_bytes_per_iteration(1000, A.nnz, ps) for ps in (8, 16, 32)]
    assert b[0] < b[1] < b[2]
