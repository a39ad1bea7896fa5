"""The allocation-free Chebyshev entry point (hs_cheb_smooth_noalloc).

Some callers cannot call cudaMalloc at the point where they smooth: a runtime
that owns the whole device memory pool, code that runs under an allocator
lock, or a serving loop that forbids allocation on its hot path.  For them the
library offers hs_cheb_smooth_noalloc: the caller passes the matrix and every
vector as device buffers it owns, and the smoother's work vectors come from a
static device array instead of cudaMalloc.

This test calls it through the C ABI and checks it against the allocating
entry point (hs_cheb_smooth on a handle built by hs_cheb_create) on two calls
in a row, so the second call runs over the array the first one left behind.
The tolerance is the one the other smoother tests use: bitwise equality.  This
file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import hsb200
from hsb200 import _lib
from hsb200 import workloads as W

pytestmark = pytest.mark.gpu


def dev(a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


@pytest.mark.parametrize("kind", [4, 1])
def test_noalloc_matches_allocating_entry_point(kind):
    A = W.poisson3d_7pt(24)                      # n = 13,824 (limit 262,144)
    n = A.shape[0]
    R = A.tocsr()
    R.sort_indices()
    cfg = (hsb200.ChebyshevFourth if kind == 4 else hsb200.ChebyshevFirst)(degree=4)
    S = hsb200.build_smoother(cfg, A)
    info = S.info
    # caller-owned device operands: CSR and l1inv = 1 ./ (l1 row sums in
    # column order, the same sums the handle computed on the device)
    l1 = np.zeros(n)
    for i in range(n):
        for q in range(R.indptr[i], R.indptr[i + 1]):
            l1[i] += abs(R.data[q])
    rp = dev(R.indptr, torch.int32)
    ci = dev(R.indices, torch.int32)
    v = dev(R.data, torch.float64)
    l1inv = dev(1.0 / l1, torch.float64)
    L = hsb200.lib()
    rng = np.random.default_rng(kind)
    for call in range(2):
        b = rng.uniform(-1, 1, n)
        x0 = rng.uniform(-1, 1, n)
        x_ref = dev(x0, torch.float64)
        x_new = dev(x0, torch.float64)
        bd = dev(b, torch.float64)
        hsb200.smooth_(x_ref, S, bd)
        st = L.hs_cheb_smooth_noalloc(n, R.nnz, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()),
                                      C.c_void_p(v.data_ptr()), C.c_void_p(l1inv.data_ptr()), kind, 4,
                                      float(info.rho), float(info.astar), C.c_void_p(x_new.data_ptr()),
                                      C.c_void_p(bd.data_ptr()), None)
        _lib.check(st)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(x_new.cpu().numpy(), x_ref.cpu().numpy(), err_msg=f"call {call}")


def test_noalloc_rejects_oversize():
    L = hsb200.lib()
    st = L.hs_cheb_smooth_noalloc(262145, 0, C.c_void_p(8), C.c_void_p(8), C.c_void_p(8), C.c_void_p(8), 4, 4,
                                  1.0, 0.0, C.c_void_p(8), C.c_void_p(8), None)
    assert st == _lib.HS_ERR_ARG
    assert b"262144" in L.hs_last_error()
