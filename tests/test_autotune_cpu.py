"""The serving tuner's decisions (hsb200/autotune.py:OnlineTuner), without a
GPU: candidates handed out in turn per class on small requests only, refused
admissions handed out again, and the partsize with the fewest modelled bytes
to convergence (iterations per n^(1/d)) kept once every candidate has
finished."""
import scipy.sparse as sp

from hsb200.autotune import OnlineTuner, batch_bytes_per_iteration, serving_class
from hsb200 import workloads as W


def test_explores_then_exploits():
    A = W.poisson2d_matrix(40)
    B = W.poisson3d_7pt(12)
    assert serving_class(A) != serving_class(B)
    t = OnlineTuner(candidates=(8, 16, 32), default=8)
    got = [t.partsize_for(A, i) for i in range(3)]
    assert got == [8, 16, 32]
    assert t.partsize_for(A, 3) == 8           # nothing finished yet: the default
    assert t.partsize_for(B, 100) == 8         # another class explores on its own
    assert t.partsize_for(B, 101) == 16
    # 16 converges in fewer modelled bytes than 8 and 32
    n, nnz = A.shape[0], A.nnz
    iters = {0: 300, 1: 100, 2: 95, 3: 300}
    for tag, it in iters.items():
        t.observe(tag, it)
    costs = {ps: iters[i] * batch_bytes_per_iteration(n, nnz, ps) for i, ps in enumerate((8, 16, 32))}
    best = min(costs, key=costs.get)
    assert best == 16 and t.choice(A) == best
    assert t.partsize_for(A, 4) == best
    assert t.partsize_for(B, 102) == 32        # B still explores


def test_large_requests_do_not_explore():
    small = W.poisson2d_matrix(30)
    big = sp.identity(1 << 18, format="csr") * 4.0 + sp.eye(1 << 18, k=1, format="csr") + \
        sp.eye(1 << 18, k=-1, format="csr")
    t = OnlineTuner(candidates=(8, 16, 32), default=8, explore_max_n=1 << 17)
    assert serving_class(big) == serving_class(small)
    assert [t.partsize_for(big, i) for i in range(3)] == [8, 8, 8]
    t.observe(0, 50)                           # a default run counts as 8's trial
    assert t.partsize_for(small, 10) == 16
    assert t.partsize_for(small, 11) == 32


def test_sizes_compare_per_n_to_the_1_over_d():
    """Iterations of a larger request count for less (scaled by n^(1/d))."""
    A = W.poisson2d_matrix(20)    # n = 400
    C = W.poisson2d_matrix(80)    # n = 6400: PCG iterations about 4x those of A
    t = OnlineTuner(candidates=(8, 16), default=8)
    assert t.partsize_for(A, 0) == 8 and t.partsize_for(C, 1) == 16
    t.observe(0, 50)
    t.observe(1, 160)   # 3.2x the iterations at 16x the rows: 16 wins per n^(1/2)
    assert t.choice(A) == 16


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
