"""Device CSR construction (hs_matrix_create): a CSC input is transposed on
the GPU by a stable sort of its row indices.  The SpMV through the resulting
CSR must equal, bitwise, the storage-order row sums over scipy's own CSR of the
same matrix -- with empty rows and columns, a single entry, FP32 storage, and
a CSR input passed through unchanged."""
import numpy as np
import pytest
import scipy.sparse as sp

torch = pytest.importorskip("torch")

import hsb200
from oracle import hs_oracle as O

pytestmark = pytest.mark.gpu


def _random_csc(n, density, seed, empty_rows=(), empty_cols=()):
    rng = np.random.default_rng(seed)
    A = sp.random(n, n, density=density, random_state=rng, format="lil")
    for r in empty_rows:
        A[r, :] = 0
    for c in empty_cols:
        A[:, c] = 0
    A = A.tocsc()
    A.eliminate_zeros()
    A.sort_indices()
    return A


@pytest.mark.parametrize("n,density", [(1, 1.0), (7, 0.5), (300, 0.03), (5000, 0.002)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_csc_transpose_spmv_bitwise(n, density, dtype):
    A = _random_csc(n, density, seed=n, empty_rows=(0, n // 2) if n > 2 else (),
                    empty_cols=(n - 1,) if n > 2 else ())
    M = hsb200.DeviceSparseMatrix(A, dtype=dtype)
    x = np.random.default_rng(1).uniform(-1, 1, n)
    xd = torch.from_numpy(x.astype(dtype)).cuda()
    y = torch.zeros_like(xd)
    hsb200.mul_(y, M, xd)
    R = A.tocsr()
    R.sort_indices()
    ref = O.spmv(R.indptr, R.indices, R.data.astype(dtype), x.astype(dtype))
    np.testing.assert_array_equal(y.cpu().numpy(), ref)


def test_csr_input_unchanged():
    A = _random_csc(400, 0.02, seed=5).tocsr()
    M = hsb200.DeviceSparseMatrix(A)
    x = np.random.default_rng(2).uniform(-1, 1, 400)
    y = torch.zeros(400, dtype=torch.float64, device="cuda")
    hsb200.mul_(y, M, torch.from_numpy(x).cuda())
    ref = O.spmv(A.indptr, A.indices, A.data, x)
    np.testing.assert_array_equal(y.cpu().numpy(), ref)
