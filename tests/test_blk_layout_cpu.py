"""CPU check of the blocked cooperative sweep's layout and order of operations
(csrc/l1gs_coop.cuh "blocked variant", csrc/l1gs_blk.cu), before any GPU
run.

The stream is built with the layout's index formulas (restated below from
hscoop::lower_idx / upper_idx), checked to be a bijection onto each group's
stream, and read back the way the kernel reads it: item by item (per row
block the off-diagonal warp tiles, then the diagonal tile), the next item's
position and kind from the kernel's state machine, each off-diagonal tile as
the lane's 16-byte vectors at `pos + lane * V + v * 32 * V`, each diagonal
entry at the kernel's offset; every read asserts that it stays inside the
group's stream and returns the intended entry.  The arithmetic is the
kernel's: dense products in column order for the off-diagonal tiles, the
diagonal solve with the solved value broadcast (forward: divided by D_Dl1 at
every step; backward and symmetric: multiplied by 1/D_Dl1), separately rounded
multiply and add, rows past n held at 0.  Forward sweeps must equal the oracle bit for
bit, backward and symmetric sweeps within 1e-12.
"""
import math

import numpy as np
import pytest

from hsb200 import workloads as W
from oracle import hs_oracle as O

B = 8
G = 4
TILE = 32 * B
DG = G * B * (B - 1) // 2


def make_layout(ps, lower, upper, es):
    psb = -(-ps // B) * B   # padded to a multiple of 8 (zero rows and columns)
    Ld = G * psb * (psb - 1) // 2
    Lg = 2 * Ld if (lower and upper) else Ld
    q = 128 // es
    return dict(ps=ps, psb=psb, G=G, V=16 // es, Ld=Ld, Lg=Lg, Lgp=(Lg + q - 1) // q * q, upper_off=Ld if lower else 0)


def lower_idx(L, k, li, lj):
    q, g = divmod(k, G)
    V = L["V"]
    I, ii = divmod(li, B)
    J, jj = divmod(lj, B)
    rs = TILE * (I * (I - 1) // 2) + I * DG
    if J < I:
        off = rs + J * TILE + (jj // V) * 32 * V + (g * B + ii) * V + jj % V
    else:
        off = rs + I * TILE + G * (jj * (B - 1) - jj * (jj - 1) // 2) + g * (B - 1 - jj) + (ii - jj - 1)
    return q * L["Lgp"] + off


def upper_idx(L, k, li, lj):
    q, g = divmod(k, G)
    V = L["V"]
    I, ii = divmod(li, B)
    J, jj = divmod(lj, B)
    m = L["psb"] // B - 1 - I
    rs = TILE * (m * (m - 1) // 2) + m * DG
    if J > I:
        off = rs + (J - I - 1) * TILE + (jj // V) * 32 * V + (g * B + ii) * V + jj % V
    else:
        off = rs + m * TILE + G * (B * (B - 1) // 2 - jj * (jj + 1) // 2) + g * jj + ii
    return q * L["Lgp"] + L["upper_off"] + off


def build_stream(A, ps, sweep, dtype):
    R = A.tocsr()
    n = A.shape[0]
    es = np.dtype(dtype).itemsize
    lower, upper = sweep != "backward", sweep != "forward"
    L = make_layout(ps, lower, upper, es)
    nparts = -(-n // ps)
    ngroups = -(-nparts // G)
    SC = np.zeros(ngroups * L["Lgp"], dtype=dtype)
    for i in range(n):
        k, li = divmod(i, ps)
        s = k * ps
        e = min(s + ps - 1, n - 1)
        for p in range(R.indptr[i], R.indptr[i + 1]):
            j = R.indices[p]
            if s <= j < i and lower:
                SC[lower_idx(L, k, li, j - s)] = R.data[p]
            elif i < j <= e and upper:
                SC[upper_idx(L, k, li, j - s)] = R.data[p]
    return L, SC, ngroups


def emulate(A, ps, sweep, D, x, dtype):
    T = np.dtype(dtype).type
    es = np.dtype(dtype).itemsize
    n = A.shape[0]
    L, SC, ngroups = build_stream(A, ps, sweep, dtype)
    owner = {}   # stream position -> (partition, row, column): what the read must return
    for k in range(ngroups * G):   # padded rows and columns too: they hold zeros
        for li in range(L["psb"]):
            for lj in range(L["psb"]):
                if lj < li and sweep != "backward":
                    owner[lower_idx(L, k, li, lj)] = (k, li, lj)
                elif lj > li and sweep != "forward":
                    owner[upper_idx(L, k, li, lj)] = (k, li, lj)
    V = L["V"]
    psb = L["psb"]
    nb = psb // B
    y = np.zeros(n, dtype=dtype)
    for q in range(ngroups):
        base = q * L["Lgp"]
        rowbase = q * G * ps
        ys = np.zeros(G * psb, dtype=dtype)

        def rd(pos, off, k, li, lj):
            assert 0 <= pos + off < L["Lg"], "read outside the group's stream"
            assert pos % V == 0, "vector read not 16-byte aligned"
            assert owner[base + pos + off] == (k, li, lj), "read of the wrong entry"
            return SC[base + pos + off]

        def tile(acc, pos, I, J):
            for lane in range(32):
                g, r = divmod(lane, B)
                for v in range(B // V):
                    for c in range(V):
                        col = v * V + c
                        a = rd(pos, v * 32 * V + lane * V + c, q * G + g, I * B + r, J * B + col)
                        acc[lane] = T(acc[lane] + T(a * ys[g * psb + J * B + col]))
            return acc

        rows = [[rowbase + g * ps + I * B + r for g, r in (divmod(l, B) for l in range(32))] for I in range(nb)]
        real = [[(I * B + l % B) < ps and rows[I][l] < n for l in range(32)] for I in range(nb)]
        with np.errstate(all="ignore"):
            if sweep != "backward":
                I, J, pos = 0, 0, 0
                acc = [T(0)] * 32
                while True:
                    is_tile = J < I
                    npos = pos + (TILE if is_tile else DG)
                    In, Jn = (I, J + 1) if is_tile else (I + 1, 0)
                    if is_tile:
                        acc = tile(acc, pos, I, J)
                    else:
                        valid = real[I]
                        xr = [T(x[rr]) if v else T(0) for rr, v in zip(rows[I], valid)]
                        dr = [D[rr] if v else T(1) for rr, v in zip(rows[I], valid)]
                        yown = [T(0)] * 32
                        rinv = [T(T(1) / dr[l]) for l in range(32)]
                        for c in range(B):
                            if sweep == "forward":   # a division at every step: bit-identical
                                v = [T((xr[l] - acc[l]) / dr[l]) for l in range(32)]
                            else:                    # symmetric: multiply by 1/D_Dl1
                                v = [T(T(xr[l] - acc[l]) * rinv[l]) for l in range(32)]
                            for lane in range(32):
                                g, r = divmod(lane, B)
                                if r == c:
                                    yown[lane] = v[lane]
                                if c < B - 1 and r > c:
                                    off = G * (c * (B - 1) - c * (c - 1) // 2) + g * (B - 1 - c) + (r - c - 1)
                                    a = rd(pos, off, q * G + g, I * B + r, I * B + c)
                                    acc[lane] = T(acc[lane] + T(a * v[g * B + c]))
                        for lane in range(32):
                            g, r = divmod(lane, B)
                            ys[g * psb + I * B + r] = yown[lane] if valid[lane] else T(0)
                        acc = [T(0)] * 32
                    if In >= nb:
                        assert npos == L["Ld"]
                        break
                    I, J, pos = In, Jn, npos
            if sweep != "forward":
                pos = L["Lg"] // 2 if sweep == "symmetric" else 0
                I, J = nb - 1, nb
                acc = [T(0)] * 32
                while True:
                    is_tile = J < nb
                    npos = pos + (TILE if is_tile else DG)
                    In, Jn = (I, J + 1) if is_tile else (I - 1, I)
                    if is_tile:
                        acc = tile(acc, pos, I, J)
                    else:
                        valid = real[I]
                        dr = [D[rr] if v else T(1) for rr, v in zip(rows[I], valid)]
                        if sweep == "symmetric":
                            xr = [T(dr[l] * ys[(l // B) * psb + I * B + l % B]) for l in range(32)]
                        else:
                            xr = [T(x[rr]) if v else T(0) for rr, v in zip(rows[I], valid)]
                        yown = [T(0)] * 32
                        rinv = [T(T(1) / dr[l]) for l in range(32)]
                        for c in range(B - 1, -1, -1):
                            v = [T(T(xr[l] - acc[l]) * rinv[l]) for l in range(32)]
                            for lane in range(32):
                                g, r = divmod(lane, B)
                                if r == c:
                                    yown[lane] = v[lane]
                                if c > 0 and r < c:
                                    off = G * (B * (B - 1) // 2 - c * (c + 1) // 2) + g * c + r
                                    a = rd(pos, off, q * G + g, I * B + r, I * B + c)
                                    acc[lane] = T(acc[lane] + T(a * v[g * B + c]))
                        for lane in range(32):
                            g, r = divmod(lane, B)
                            ys[g * psb + I * B + r] = yown[lane] if valid[lane] else T(0)
                        acc = [T(0)] * 32
                    if In < 0:
                        assert npos == L["Lg"]
                        break
                    I, J, pos = In, Jn, npos
        for t in range(G * psb):
            pp, li = divmod(t, psb)
            if li < ps and rowbase + pp * ps + li < n:
                y[rowbase + pp * ps + li] = ys[t]
    return y


@pytest.mark.parametrize("ps", [8, 16, 31, 32, 64])
def test_blk_layout_is_a_bijection(ps):
    """Every strict-triangle slot of every partition maps to a distinct entry
    of its group's stream, and the stream has no holes."""
    for es in (8, 4):
        for lower, upper in ((True, False), (False, True), (True, True)):
            L = make_layout(ps, lower, upper, es)
            seen = set()
            for k in range(2 * G):
                for li in range(L["psb"]):
                    for lj in range(L["psb"]):
                        if lj < li and lower:
                            p = lower_idx(L, k, li, lj)
                        elif lj > li and upper:
                            p = upper_idx(L, k, li, lj)
                        else:
                            continue
                        assert p not in seen
                        seen.add(p)
                        q = k // G
                        assert q * L["Lgp"] <= p < q * L["Lgp"] + L["Lg"]
            assert len(seen) == 2 * L["Lg"]


@pytest.mark.parametrize("ps,n", [(8, 77), (16, 150), (24, 333), (32, 300), (40, 257), (64, 500), (128, 700),
                                  (12, 200), (31, 500), (33, 400), (100, 1000)])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_blk_emulation_matches_oracle(ps, n, sweep):
    A = W.poisson2d_matrix(int(math.ceil(math.sqrt(n))), eps=0.3)
    A = A[:n, :n].tocsc()
    A.sort_indices()
    rng = np.random.default_rng(ps + n)
    A.data = A.data * rng.uniform(0.5, 1.5, A.nnz)   # distinct values: a misplaced entry shows
    x = rng.uniform(-1, 1, n)
    ref = O.OracleL1GS(A, ps, isSymA=False, sweep=sweep, cache="packed")
    want = ref.ldiv(x)
    got = emulate(A, ps, sweep, ref.D, x, np.float64)
    if sweep == "forward":
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_blk_emulation_fp32_and_nonfinite():
    A = W.poisson2d_matrix(18, eps=0.3).astype(np.float32)
    n = A.shape[0]
    x = np.random.default_rng(1).uniform(-1, 1, n).astype(np.float32)
    x[[5, 100, 200]] = [np.inf, np.nan, -np.inf]
    for sweep in ("forward", "symmetric"):
        ref = O.OracleL1GS(A, 24, isSymA=True, sweep=sweep, cache="packed")
        with np.errstate(all="ignore"):
            want = ref.ldiv(x)
        got = emulate(A, 24, sweep, ref.D, x, np.float32)
        if sweep == "forward":
            np.testing.assert_array_equal(got, want)
        else:
            fin = np.isfinite(want)
            np.testing.assert_array_equal(np.isfinite(got), fin)
            np.testing.assert_allclose(got[fin], want[fin], rtol=1e-5, atol=1e-5 * np.abs(want[fin]).max())


class ItemCursor:
    """hscoop::ItemCursor (csrc/l1gs_blk.cu): the copy side's walk over a
    warp's items, run ahead of the arithmetic."""

    def __init__(self, sweep, q0, qstride, gend, nb, Lg):
        self.sweep, self.qstride, self.gend, self.nb, self.Lg = sweep, qstride, gend, nb, Lg
        self.start_group(q0)

    def start_group(self, q):
        self.q, self.valid = q, q < self.gend
        if self.sweep == "backward":
            self.dir, self.I, self.J = 1, self.nb - 1, self.nb
        else:
            self.dir, self.I, self.J = 0, 0, 0
        self.pos = 0

    def is_tile(self):
        return self.J < self.I if self.dir == 0 else self.J < self.nb

    def advance(self):
        t = self.is_tile()
        self.pos += TILE if t else DG
        if self.dir == 0:
            if t:
                self.J += 1
            else:
                self.I, self.J = self.I + 1, 0
                if self.I == self.nb:
                    if self.sweep == "symmetric":
                        self.dir, self.I, self.J, self.pos = 1, self.nb - 1, self.nb, self.Lg // 2
                    else:
                        self.start_group(self.q + self.qstride)
        else:
            if t:
                self.J += 1
            else:
                self.I -= 1
                if self.I < 0:
                    self.start_group(self.q + self.qstride)
                else:
                    self.J = self.I + 1


def consumer_items(sweep, q0, qstride, gend, nb, Lg):
    """The arithmetic side's item order: (group, position, is tile, J)."""
    out = []
    for q in range(q0, gend, qstride):
        if sweep != "backward":
            pos = 0
            for I in range(nb):
                for J in range(I):
                    out.append((q, pos, True, J))
                    pos += TILE
                out.append((q, pos, False, I))
                pos += DG
            assert pos == (Lg // 2 if sweep == "symmetric" else Lg)
        if sweep != "forward":
            pos = Lg // 2 if sweep == "symmetric" else 0
            for I in range(nb - 1, -1, -1):
                for J in range(I + 1, nb):
                    out.append((q, pos, True, J))
                    pos += TILE
                out.append((q, pos, False, I))
                pos += DG
            assert pos == Lg
    return out


@pytest.mark.parametrize("ps", [8, 16, 64])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_blk_copy_cursor_matches_arithmetic(ps, sweep):
    """The copies (kRing - 1 items ahead, one commit group per item, empty
    groups past the end) land every item the arithmetic reads, in its order,
    into the slot it reads, and never overwrite a slot still to be read."""
    kring = 4
    nb = ps // B
    L = make_layout(ps, sweep != "backward", sweep != "forward", 8)
    for q0, qstride, gend in ((0, 3, 7), (2, 3, 3), (5, 3, 4)):
        want = consumer_items(sweep, q0, qstride, gend, nb, L["Lg"])
        ic = ItemCursor(sweep, q0, qstride, gend, nb, L["Lg"])
        groups = []   # commit groups in order: the item each copied, or None (empty)
        slots = {}

        def issue(slot):
            if ic.valid:
                groups.append((ic.q, ic.pos, ic.is_tile()))
                slots[slot] = len(groups) - 1
                ic.advance()
            else:
                groups.append(None)
        for s in range(kring - 1):
            issue(s)
        for k, (q, pos, is_tile, _) in enumerate(want):
            # wait_group(kring - 2): groups 0..k have completed
            assert len(groups) == k + kring - 1
            issue((k + kring - 1) % kring)
            assert slots[k % kring] == k, "slot overwritten before it was read"
            assert groups[k] == (q, pos, is_tile)
        assert not ic.valid and all(gr is None for gr in groups[len(want):])
