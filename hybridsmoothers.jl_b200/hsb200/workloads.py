"""Seeded synthetic matrices and right-hand sides for the five workloads of
the HybridSmoothers.jl smoother path, plus the reference's own test matrices.

Reference test fixtures restated (test/test_matrices.jl:5-19):
  poisson_test_matrix(N), poisson2d_matrix(n; eps), convection_diffusion_matrix(n; eps, c).

Benchmark workloads (no public suite exists; all are generated here):
  1. 1D Laplacian N=2048 (diag 2, off-diagonal -1), b = ones.
  2. 3D 7-point Poisson on 128^3, Dirichlet (kron of the 1D (2,-1) operator in
     three directions: diag 6, off-diagonal -1), b ~ U[-1, 1].
  3. 3D upwind convection-diffusion on 96^3: 7-point Laplacian scaled by 1/h^2
     plus first-order upwind differences for the velocity (1, 0.5, 0.25)*Pe,
     Pe = 10, h = 1/97 (grid Peclet number Pe*h/2 per direction).
  4. 3D 27-point anisotropic variable-coefficient diffusion on 160^3: a graph
     Laplacian over the 26-neighbourhood with Dirichlet closure, edge weight
     = (direction factor) * sqrt(k_i k_j), k ~ lognormal(0, sigma=1) per cell,
     direction factors (1, 0.3, 0.1) for x/y/z faces, edges the mean of their
     two axes' factors times 1/2, corners the mean of three times 1/4.
  5. Serving stream: 2D 5-point or 3D 7-point diffusion with per-edge
     coefficients U[0.1, 10], sizes log-uniform in [1e3, 2e6].

All generators return scipy CSC matrices with sorted indices (CSC == CSR
structure for the symmetric ones), int32 indices and float64 values.
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

SEED = 20261203


# ---------------------------------------------------------------------------
# Reference test matrices (test/test_matrices.jl)
# ---------------------------------------------------------------------------

def poisson_test_matrix(N):
    """spdiagm(0 => 2 ones(N), -1 => -ones(N-1), 1 => -ones(N-1)), CSC."""
    A = sp.diags([-np.ones(N - 1), 2 * np.ones(N), -np.ones(N - 1)], [-1, 0, 1], format="csc")
    return _canon(A)


def poisson2d_matrix(n, eps=1.0):
    T = poisson_test_matrix(n)
    I = sp.identity(n, format="csc")
    return _canon(sp.kron(I, T) + eps * sp.kron(T, I))


def convection_diffusion_matrix(n, eps=1.0, c=1.0):
    upwind = sp.diags([np.ones(n), -np.ones(n - 1)], [0, -1], format="csc")
    return _canon(poisson2d_matrix(n, eps) + c * sp.kron(sp.identity(n, format="csc"), upwind))


def _canon(A, fmt="csc"):
    A = A.asformat(fmt)
    A.sum_duplicates()
    A.sort_indices()
    A.indptr = A.indptr.astype(np.int32)
    A.indices = A.indices.astype(np.int32)
    A.data = A.data.astype(np.float64)
    return A


# ---------------------------------------------------------------------------
# Structured-grid stencil assembly (vectorised, sorted columns per row)
# ---------------------------------------------------------------------------

def _stencil_csr(shape, offsets, values):
    """Assemble a CSR matrix from a structured-grid stencil.

    shape: (nz, ny, nx) with x fastest; offsets: list of (dz, dy, dx);
    values: list of arrays of shape (nz, ny, nx) giving the coefficient that
    row p puts on column p+offset (ignored where the neighbour is outside).
    Offsets are sorted by linear offset so each row's columns come out
    ascending.
    """
    nz, ny, nx = shape
    N = nz * ny * nx
    lin = [dz * ny * nx + dy * nx + dx for dz, dy, dx in offsets]
    order = np.argsort(lin)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    masks, cols, vals = [], [], []
    base = np.arange(N, dtype=np.int64).reshape(shape)
    for o in order:
        dz, dy, dx = offsets[o]
        m = (z + dz >= 0) & (z + dz < nz) & (y + dy >= 0) & (y + dy < ny) & (x + dx >= 0) & (x + dx < nx)
        masks.append(m.ravel())
        cols.append((base + lin[o]).ravel())
        vals.append(np.broadcast_to(values[o], shape).ravel())
    M = np.stack(masks, axis=1)           # N x K
    counts = M.sum(axis=1)
    indptr = np.zeros(N + 1, dtype=np.int64)
    np.cumsum(counts, out=indptr[1:])
    Cc = np.stack(cols, axis=1)[M]
    Vv = np.stack(vals, axis=1)[M]
    A = sp.csr_matrix((Vv.astype(np.float64), Cc.astype(np.int32), indptr.astype(np.int32)), shape=(N, N))
    A.has_sorted_indices = True
    return A


def poisson3d_7pt(n):
    """Workload 2: 7-point Poisson on n^3 with Dirichlet boundaries (diag 6, off -1)."""
    shape = (n, n, n)
    offs = [(0, 0, 0), (-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)]
    vals = [np.float64(6.0)] + [np.float64(-1.0)] * 6
    A = _stencil_csr(shape, offs, vals)
    # symmetric: the CSR arrays are also the CSC arrays
    return _canon(sp.csc_matrix((A.data, A.indices, A.indptr), shape=A.shape))


def convdiff3d_upwind(n=96, Pe=10.0, vel=(1.0, 0.5, 0.25)):
    """Workload 3: non-symmetric upwind convection-diffusion on n^3, h = 1/(n+1)."""
    h = 1.0 / (n + 1)
    vx, vy, vz = (Pe * v for v in vel)
    inv_h2 = 1.0 / (h * h)
    # Laplacian part: 6/h^2 on the diagonal, -1/h^2 to each face neighbour.
    # Upwind first differences for positive velocity components:
    #   v * (u_p - u_{p-1}) / h  ->  +v/h on the diagonal, -v/h on the upstream neighbour.
    diag = 6.0 * inv_h2 + (vx + vy + vz) / h
    offs = [(0, 0, 0), (0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)]
    vals = [diag,
            -inv_h2 - vx / h, -inv_h2,
            -inv_h2 - vy / h, -inv_h2,
            -inv_h2 - vz / h, -inv_h2]
    vals = [np.float64(v) for v in vals]
    A = _stencil_csr((n, n, n), offs, vals)
    return _canon(A, "csc")


def aniso27_lognormal(n=160, sigma=1.0, seed=SEED, factors=(1.0, 0.3, 0.1)):
    """Workload 4: 27-point anisotropic lognormal-coefficient diffusion on n^3."""
    rng = np.random.default_rng(seed)
    shape = (n, n, n)
    k = np.exp(sigma * rng.standard_normal(shape))
    sk = np.sqrt(k)
    fx, fy, fz = factors
    offs, vals = [], []
    diag = np.zeros(shape)
    for dz in (-1, 0, 1):
        for dy in (-1, 0, 1):
            for dx in (-1, 0, 1):
                if dz == 0 and dy == 0 and dx == 0:
                    continue
                axes = [f for f, d in zip((fz, fy, fx), (dz, dy, dx)) if d != 0]
                nax = len(axes)
                w_dir = float(np.mean(axes)) * {1: 1.0, 2: 0.5, 3: 0.25}[nax]
                # neighbour coefficient; outside the grid the cell's own value is used
                # and the edge survives only on the diagonal (Dirichlet closure)
                src = [slice(None)] * 3
                dst = [slice(None)] * 3
                for ax, d in enumerate((dz, dy, dx)):
                    if d == 1:
                        dst[ax] = slice(0, n - 1); src[ax] = slice(1, n)
                    elif d == -1:
                        dst[ax] = slice(1, n); src[ax] = slice(0, n - 1)
                nbk = sk.copy()
                nbk[tuple(dst)] = sk[tuple(src)]
                w = w_dir * (sk * nbk)   # sk*nbk is commutative, so A is exactly symmetric
                offs.append((dz, dy, dx))
                vals.append(-w)
                diag += w
    offs.append((0, 0, 0))
    vals.append(diag)
    A = _stencil_csr(shape, offs, vals)
    return _canon(sp.csc_matrix((A.data, A.indices, A.indptr), shape=A.shape))


def variable_diffusion(dims, rng):
    """Workload 5 member: 2D 5-point or 3D 7-point, per-edge coefficients U[0.1, 10]."""
    if len(dims) == 2:
        shape = (1,) + tuple(dims)
        axes = [(0, 1, 0), (0, 0, 1)]
    else:
        shape = tuple(dims)
        axes = [(1, 0, 0), (0, 1, 0), (0, 0, 1)]
    nz, ny, nx = shape
    diag = np.zeros(shape)
    offs, vals = [], []
    for d in axes:
        w = rng.uniform(0.1, 10.0, size=shape)   # edge between p and p+d
        # p -> p+d uses w[p]; p -> p-d uses w[p-d]
        wm = np.zeros(shape)
        src = [slice(None)] * 3
        dst = [slice(None)] * 3
        for ax, dd in enumerate(d):
            if dd:
                dst[ax] = slice(1, shape[ax]); src[ax] = slice(0, shape[ax] - 1)
        wm[tuple(dst)] = w[tuple(src)]
        # boundary edges (neighbour outside) act as Dirichlet closures on the diagonal
        diag += w + np.where(wm > 0, wm, rng.uniform(0.1, 10.0, size=shape))
        offs += [d, tuple(-x for x in d)]
        vals += [-w, -wm]
    offs.append((0, 0, 0))
    vals.append(diag)
    A = _stencil_csr(shape, offs, vals)
    A = (A + A.T) * 0.5   # exact symmetry of the assembled values
    return _canon(A, "csc")


def serving_stream(count=512, lo=1e3, hi=2e6, seed=SEED, rate=None):
    """Workload 5: (arrival_time_s, matrix, rhs) triples, Poisson arrivals."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    for _ in range(count):
        size = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        if rng.random() < 0.5:
            s = max(4, int(round(size ** 0.5)))
            dims = (s, s)
        else:
            s = max(3, int(round(size ** (1.0 / 3.0))))
            dims = (s, s, s)
        A = variable_diffusion(dims, rng)
        b = rng.uniform(-1.0, 1.0, size=A.shape[0])
        if rate is not None:
            t += rng.exponential(1.0 / rate)
        out.append((t, A, b))
    return out


def rhs_uniform(n, seed=SEED):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=n)
