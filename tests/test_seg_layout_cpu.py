"""CPU check of the matrix-view sweep over segment lists
(csrc/l1gs_seg.cuh, csrc/l1gs_seg.cu), before any GPU run.

The emulation builds the per-group streams with the build kernels' formulas
(in-block counts, per-row maximum over the group's 32 partitions, row offsets
in the sweep's order, group bases, padding slots holding 0 and the column
`ps`), then runs the apply lane by lane: the warp's chunks are "copied" into
a 4-stage ring in issue order, each read asserts that its chunk has landed
and has not been released, finished chunks are released inside a row, the
slot position is a running (chunk, slot) pair, and every lane runs all of
the row's slots -- its padding adds 0 * y[ps] with y[ps] = +0.  Results must
equal the oracle's view path bit for bit, non-finite inputs included.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from hsb200 import workloads as W
from oracle import hs_oracle as O


def build(A_rows, ps, dtype, G=32):
    R = A_rows
    n = R.shape[0]
    nparts = -(-n // ps)
    ngroups = -(-nparts // G)
    cntL = np.zeros(n, int)
    qL = np.zeros(n, int)
    cntU = np.zeros(n, int)
    qU = np.zeros(n, int)
    for i in range(n):
        s = (i // ps) * ps
        e = min(s + ps - 1, n - 1)
        q0, q1 = R.indptr[i], R.indptr[i + 1]
        ql = qu = q0
        cl = cu = 0
        for q in range(q0, q1):
            j = R.indices[q]
            if s <= j < i:
                if cl == 0:
                    ql = q
                cl += 1
            elif i < j <= e:
                if cu == 0:
                    qu = q
                cu += 1
        cntL[i], qL[i], cntU[i], qU[i] = cl, ql, cu, qu
    dirs = {}
    for name, cnt, q0, desc in (("lo", cntL, qL, False), ("up", cntU, qU, True)):
        maxc = np.zeros((ngroups, ps), int)
        cnti = np.zeros((ngroups, ps, G), int)
        for g in range(ngroups):
            for li in range(ps):
                vals = []
                for lane in range(G):
                    k = g * G + lane
                    row = k * ps + li
                    c = cnt[row] if (k < nparts and row < n) else 0
                    cnti[g, li, lane] = c
                    vals.append(c)
                maxc[g, li] = max(vals)
        off = np.zeros((ngroups, ps), int)
        total = np.zeros(ngroups, int)
        for g in range(ngroups):
            acc = 0
            for t in range(ps):
                li = ps - 1 - t if desc else t
                off[g, li] = acc
                acc += maxc[g, li]
            total[g] = acc
        base = np.concatenate([[0], np.cumsum(total)[:-1]]).astype(int)
        slots = int(total.sum())
        vals = np.zeros((slots, G), dtype=dtype)
        cols = np.full((slots, G), ps, dtype=np.int64)
        for i in range(n):
            k, li = divmod(i, ps)
            g, lane = divmod(k, G)
            s = k * ps
            for t in range(cnt[i]):
                q = q0[i] + t
                slot = base[g] + off[g, li] + t
                vals[slot, lane] = R.data[q]
                cols[slot, lane] = R.indices[q] - s
        dirs[name] = dict(maxc=maxc, cnti=cnti, off=off, total=total, base=base, vals=vals, cols=cols)
    return dirs, ngroups


class Ring:
    def __init__(self, chunks, nst=4):
        self.chunks = chunks     # list of (dir, first slot) per virtual chunk, issue order
        self.nst = nst
        self.owner = [-1] * nst
        self.issued = self.ready = self.freed = 0
        self.fill()

    def fill(self):
        while self.issued < len(self.chunks) and self.issued < self.freed + self.nst:
            s = self.issued % self.nst
            assert self.owner[s] < self.freed, "stage refilled before its chunk was released"
            self.owner[s] = self.issued
            self.issued += 1

    def wait_upto(self, last):
        while self.ready <= last:
            assert self.ready < self.issued, "wait on a chunk never issued (the kernel would time out)"
            self.ready += 1

    def release(self, upto):
        if upto > self.freed:
            self.freed = upto
            self.fill()

    def check(self, c):
        assert self.owner[c % self.nst] == c and self.freed <= c < self.ready


def emulate(A_rows, ps, sweep, D, x, dtype, warps=2, K=None, G=32):
    T = np.dtype(dtype).type
    if K is None:   # slots per chunk of the kernels: 4 (FP64), 6 (FP32), times 32 / G
        K = (4 if np.dtype(dtype).itemsize == 8 else 6) * (32 // G)
    dirs, ngroups = build(A_rows, ps, dtype, G)
    n = A_rows.shape[0]
    order = {"forward": ["lo"], "backward": ["up"], "symmetric": ["lo", "up"]}[sweep]
    y = np.zeros(n, dtype=dtype)
    for w in range(warps):
        groups = list(range(w, ngroups, warps))
        chunks = []
        for g in groups:
            for d in order:
                nch = -(-int(dirs[d]["total"][g]) // K)
                chunks += [(d, g, c) for c in range(nch)]
        ring = Ring(chunks)
        ch = 0
        for g in groups:
            ys = np.zeros((ps + 1, G), dtype=dtype)   # row ps: the padding slots' target, +0
            ds = np.ones((ps, G), dtype=dtype)
            for lane in range(G):
                for li in range(ps):
                    row = (g * G + lane) * ps + li
                    if row < n:
                        ys[li, lane] = T(x[row])
                        ds[li, lane] = D[row]
            for d in order:
                dd = dirs[d]
                start = ch
                wi = 0
                o = 0      # running slot offset of the row (the stored offsets, recomputed)
                rows = range(ps) if d == "lo" else range(ps - 1, -1, -1)
                with np.errstate(all="ignore"):
                    for li in rows:
                        m = dd["maxc"][g, li]
                        assert dd["off"][g, li] == o
                        acc = np.zeros(G, dtype=dtype)
                        for k in range(m):
                            assert (ch - start) * K + wi == o + k
                            ring.wait_upto(ch)
                            ring.check(ch)
                            a = dd["vals"][dd["base"][g] + o + k]
                            col = dd["cols"][dd["base"][g] + o + k]
                            acc = acc + a * ys[col, np.arange(G)]
                            wi += 1
                            if wi == K:
                                wi = 0
                                ch += 1
                                ring.release(ch)
                        o += m
                        yi = ys[li].copy()
                        if sweep == "symmetric" and d == "up":
                            yi = ds[li] * yi
                        ys[li] = (yi - acc) / ds[li]
                if wi > 0:
                    ch += 1
                    ring.release(ch)
                assert ch - start == -(-int(dd["total"][g]) // K)
            for lane in range(G):
                for li in range(ps):
                    row = (g * G + lane) * ps + li
                    if row < n:
                        y[row] = ys[li, lane]
        assert ring.ready == ring.issued == len(chunks)
    return y


def rows_of(A, isSym):
    R = (A if isSym else A.tocsr()) if A.format == "csr" else (A.tocsr() if not isSym else A)
    if isSym and A.format == "csc":   # isSymA reads column i as row i
        R = sp.csr_matrix((A.data, A.indices, A.indptr), shape=A.shape)
    R.sort_indices()
    return R


@pytest.mark.parametrize("ps,n", [(2, 40), (5, 301), (16, 1000), (17, 999), (40, 900), (64, 1500)])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_seg_emulation_bitwise(ps, n, sweep):
    rng = np.random.default_rng(ps + n)
    A = sp.random(n, n, density=min(0.5, 12.0 / n), random_state=rng, format="csc")
    A.data = rng.uniform(-1, 1, A.nnz)
    A = A + sp.diags(rng.uniform(3, 5, n) + abs(A).sum(axis=1).A.ravel())
    A = W._canon(A.tocsc())
    x = rng.uniform(-1, 1, n)
    for fmt, isSym in (("csr", False), ("csc", True)):
        M = A.asformat(fmt)
        ref = O.OracleL1GS(M, ps, isSymA=isSym, sweep=sweep, cache="view")
        got = emulate(rows_of(M, isSym), ps, sweep, ref.D, x, np.float64)
        np.testing.assert_array_equal(got, ref.ldiv(x))


def test_seg_emulation_stencil_fp32():
    A = W.poisson3d_7pt(12).astype(np.float32)
    x = np.random.default_rng(3).uniform(-1, 1, A.shape[0]).astype(np.float32)
    ref = O.OracleL1GS(A, 16, isSymA=True, sweep="symmetric", cache="view")
    got = emulate(rows_of(A, True), 16, "symmetric", ref.D, x, np.float32)
    np.testing.assert_array_equal(got, ref.ldiv(x))


@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_seg_emulation_nonfinite(sweep):
    """Padding slots add 0 * y[ps] with y[ps] = +0: a lane whose own rows
    are shorter than the group's maximum must not pick up an inf or NaN of
    another row (0 * inf would be NaN)."""
    rng = np.random.default_rng(7)
    n, ps = 700, 16
    A = sp.random(n, n, density=8.0 / n, random_state=rng, format="csc")
    A.data = rng.uniform(-1, 1, A.nnz)
    A = A + sp.diags(rng.uniform(3, 5, n) + abs(A).sum(axis=1).A.ravel())
    A = W._canon(A.tocsc())
    x = rng.uniform(-1, 1, n)
    x[[3, 40, 41, 333]] = [np.inf, -np.inf, np.nan, np.inf]
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="view")
    with np.errstate(all="ignore"):
        want = ref.ldiv(x)
    got = emulate(rows_of(A, True), ps, sweep, ref.D, x, np.float64)
    np.testing.assert_array_equal(got, want)


def pick_group(ps, es):
    """hsseg::pick_group: the largest of 32, 16, 8, 4 with y and D_Dl1 of a
    group in at most 24 KiB."""
    G = 32
    while G > 4 and (2 * ps + 1) * (G + 1) * es > 24 * 1024:
        G //= 2
    return G


@pytest.mark.parametrize("ps,n", [(64, 3000), (128, 3000), (256, 5000), (300, 4000), (512, 6000)])
@pytest.mark.parametrize("sweep", ["forward", "symmetric"])
def test_seg_emulation_small_groups(ps, n, sweep):
    """Groups of fewer than 32 partitions (large partsizes)."""
    G = pick_group(ps, 8)
    assert G < 32
    A = W.poisson2d_matrix(int(np.ceil(np.sqrt(n))), eps=0.3)
    A = W._canon(A[:n, :n].tocsc())
    x = np.random.default_rng(ps).uniform(-1, 1, n)
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="view")
    got = emulate(rows_of(A, True), ps, sweep, ref.D, x, np.float64, G=G)
    np.testing.assert_array_equal(got, ref.ldiv(x))


def slot_bytes(G, es):
    """hsseg::slot_bytes: [G values][G uint16 columns], padded to 16 bytes."""
    return -(-(G * (es + 2)) // 16) * 16


def test_seg_copies_are_legal_bulk_copies():
    """Every slot, chunk and ring stage of the segment-list kernels starts on
    a 16-byte boundary and is a multiple of 16 bytes long, for every
    partsize the kernels take and both value types (a 1D bulk copy needs
    both)."""
    for es in (8, 4):
        K0 = 4 if es == 8 else 6
        for ps in range(2, 513):
            G = pick_group(ps, es)
            assert G in (32, 16, 8, 4)
            SB = slot_bytes(G, es)
            assert SB % 16 == 0 and SB >= G * (es + 2)
            K = K0 * (32 // G)
            CHB = K * SB
            assert CHB % 16 == 0
            for slots in range(1, K + 1):   # the last, partial chunk of a pair
                assert (slots * SB) % 16 == 0
