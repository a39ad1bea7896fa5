"""CPU check of the cooperative packed sweep's layout, ring protocol and order
of operations (csrc/l1gs_coop.cuh, csrc/l1gs_coop_kernel.cuh), before any GPU
run.

The emulation below follows the kernel lane by lane: the coop-layout stream is
built with the setup kernel's index formulas, chunks of it are "copied" into a
per-warp ring (and its tail slots) in the kernel's issue order, every ring read
uses the kernel's linear address expression and asserts that it stays inside
the ring, that its chunk has landed and has not been released, and that it
returns the intended stream entry; the arithmetic is the kernel's
(right-looking, separately rounded multiply and add).  Results are compared with the oracle: forward
sweeps bitwise, backward/symmetric to 1e-12.  No GPU is used.
"""
import math

import numpy as np
import pytest

from hsb200 import workloads as W
from oracle import hs_oracle as O


def make_layout(ps, tpp, lower, upper, es):
    G = 32 // tpp
    Ld = G * ps * (ps - 1) // 2
    Lg = 2 * Ld if (lower and upper) else Ld
    q = 128 // es
    Lgp = (Lg + q - 1) // q * q
    return dict(ps=ps, G=G, Ld=Ld, Lg=Lg, Lgp=Lgp, upper_off=Ld if lower else 0)


def colbase(ps, G, t):
    return G * (t * (ps - 1) - t * (t - 1) // 2)


def lower_idx(L, k, li, lj):
    q, g = divmod(k, L["G"])
    return q * L["Lgp"] + colbase(L["ps"], L["G"], lj) + (li - lj - 1) * L["G"] + g


def upper_idx(L, k, li, lj):
    q, g = divmod(k, L["G"])
    return q * L["Lgp"] + L["upper_off"] + colbase(L["ps"], L["G"], L["ps"] - 1 - lj) + li * L["G"] + g


def ring_geometry(ps, G, es):
    """hscoop::make_geometry: chunk size, stages, tail stages."""
    che = 2048 // es
    maxcol = G * (ps - 1)
    ntail = max(1, -(-maxcol // che))
    st = 4
    while st < ntail + 3:
        st *= 2
    return che, st, ntail


def build_stream(A, ps, tpp, sweep, dtype):
    """The setup kernel's scatter of the in-block entries into the coop layout."""
    R = A.tocsr()
    n = A.shape[0]
    es = np.dtype(dtype).itemsize
    lower, upper = sweep != "backward", sweep != "forward"
    L = make_layout(ps, tpp, lower, upper, es)
    nparts = -(-n // ps)
    ngroups = -(-nparts // L["G"])
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


class Ring:
    """One warp's ring: chunks of `che` entries in `st` stages plus `ntail`
    tail slots repeating stages 0..ntail-1; bulk copies in issue order."""

    def __init__(self, SC, L, groups, che, st, ntail, es):
        self.SC, self.L, self.groups, self.che, self.st, self.ntail = SC, L, groups, che, st, ntail
        self.nchg = -(-L["Lg"] // che)
        self.total = len(groups) * self.nchg
        self.buf = np.full(che * (st + ntail), np.nan, dtype=SC.dtype)
        self.owner = np.full(st, -1)      # chunk held by each stage
        self.src = {}                     # chunk -> stream offset of its entry 0
        self.issued = self.ready = self.freed = 0
        self.es = es
        self.fill()

    def fill(self):
        while self.issued < self.total and self.issued < self.freed + self.st:
            c = self.issued
            gi, pc = divmod(c, self.nchg)
            grp = self.groups[gi]
            off = pc * self.che
            cnt = min(self.che, self.L["Lg"] - off)
            nbytes = (cnt * self.es + 15) // 16 * 16
            src0 = grp * self.L["Lgp"] + off
            assert src0 + nbytes // self.es <= len(self.SC), "bulk copy past the stream buffer"
            assert (src0 * self.es) % 16 == 0 and nbytes % 16 == 0
            s = c % self.st
            assert self.owner[s] < 0 or self.owner[s] < self.freed, "stage refilled before it was consumed"
            slots = [s] + ([self.st + s] if s < self.ntail else [])
            for d in slots:
                self.buf[d * self.che:(d + 1) * self.che] = np.nan
                self.buf[d * self.che:d * self.che + nbytes // self.es] = self.SC[src0:src0 + nbytes // self.es]
            self.owner[s] = c
            self.src[c] = src0
            self.issued += 1

    def wait_upto(self, last):
        while self.ready <= last:
            assert self.ready < self.issued, "wait on a chunk that was never issued (the kernel would time out)"
            self.ready += 1

    def release(self, upto):
        if upto > self.freed:
            self.freed = upto
            self.fill()

    def read(self, col, idx, want_pos):
        """Entry idx of the column block whose ring position is `col` (the
        kernel's linear read); want_pos is its position in the stream."""
        addr = (col & 0xFFFFFFFF & (self.che * self.st - 1)) + idx
        assert 0 <= addr < self.che * (self.st + self.ntail), "ring read outside the linear buffer"
        slot = addr // self.che
        s = slot if slot < self.st else slot - self.st
        assert slot < self.st or s < self.ntail
        c = self.owner[s]
        assert c >= 0 and c < self.ready and c >= self.freed, "ring read of a chunk not landed or already released"
        assert self.src[c] + addr % self.che == want_pos, "ring read of the wrong stream entry"
        return self.buf[addr]


def emulate(A, ps, tpp, sweep, D, x, dtype, warps=3):
    """The kernel's arithmetic and ring traffic, lane by lane, on `warps` warps
    that take groups q0, q0 + warps, ..."""
    T = np.dtype(dtype).type
    n = A.shape[0]
    es = np.dtype(dtype).itemsize
    L, SC, ngroups = build_stream(A, ps, tpp, sweep, dtype)
    G = L["G"]
    M = -(-ps // tpp)
    che, st, ntail = ring_geometry(ps, G, es)
    l2 = int(math.log2(che))
    y = np.zeros(n, dtype=dtype)
    lanes = np.arange(32)
    g_of, r_of = lanes // tpp, lanes % tpp
    for w in range(warps):
        groups = list(range(w, ngroups, warps))
        ring = Ring(SC, L, groups, che, st, ntail, es)
        for gi, q in enumerate(groups):
            c0 = gi * ring.nchg
            vg = (c0 << l2) & 0xFFFFFFFF
            yv = np.zeros((32, M), dtype=dtype)
            dv = np.ones((32, M), dtype=dtype)
            acc = np.zeros((32, M), dtype=dtype)
            valid = np.zeros((32, M), dtype=bool)
            for ln in range(32):
                row0 = (q * G + g_of[ln]) * ps
                for m in range(M):
                    li = r_of[ln] + tpp * m
                    row = row0 + li
                    if li < ps and row < n:
                        valid[ln, m] = True
                        yv[ln, m] = T(x[row])
                        dv[ln, m] = D[row]
            lpos = 0
            if sweep != "backward":
                for t in range(ps):
                    mb, tr = divmod(t, tpp)
                    ln_len = ps - 1 - t
                    if ln_len > 0:
                        ring.wait_upto(c0 + ((lpos + G * ln_len - 1) >> l2))
                    v = (yv[:, mb] - acc[:, mb]) / dv[:, mb]
                    yt = np.array([v[g * tpp + tr] for g in g_of], dtype=dtype)
                    own = r_of == tr
                    yv[own, mb] = yt[own]
                    for ln in range(32):
                        r, g = r_of[ln], g_of[ln]
                        for m in range(mb, M):
                            if (m > mb or r > tr) and r + tpp * m < ps:
                                idx = (r - tr - 1) * G + g + 32 * (m - mb)
                                a = ring.read(vg + lpos, idx, q * L["Lgp"] + lpos + idx)
                                acc[ln, m] = acc[ln, m] + a * yt[ln]
                    lpos += G * ln_len
                    ring.release(c0 + (lpos >> l2))
            if sweep == "symmetric":
                yv = np.where(valid, dv * yv, T(0)).astype(dtype)
                acc[:] = 0
            if sweep != "forward":
                for j in range(ps - 1, -1, -1):
                    mb, tr = divmod(j, tpp)
                    if j > 0:
                        ring.wait_upto(c0 + ((lpos + G * j - 1) >> l2))
                    v = (yv[:, mb] - acc[:, mb]) / dv[:, mb]
                    yj = np.array([v[g * tpp + tr] for g in g_of], dtype=dtype)
                    own = r_of == tr
                    yv[own, mb] = yj[own]
                    for ln in range(32):
                        r, g = r_of[ln], g_of[ln]
                        for m in range(0, mb + 1):
                            if m < mb or r < tr:
                                idx = r * G + g + 32 * m
                                a = ring.read(vg + lpos, idx, q * L["Lgp"] + lpos + idx)
                                acc[ln, m] = acc[ln, m] + a * yj[ln]
                    lpos += G * j
                    ring.release(c0 + (lpos >> l2))
            ring.release(c0 + ring.nchg)
            for ln in range(32):
                row0 = (q * G + g_of[ln]) * ps
                for m in range(M):
                    if valid[ln, m]:
                        y[row0 + r_of[ln] + tpp * m] = yv[ln, m]
        assert ring.ready == ring.issued == ring.total, "copies left in flight at kernel exit"
    return y


@pytest.mark.parametrize("ps,tpp,n", [(16, 4, 100), (32, 4, 333), (33, 16, 200), (40, 16, 301), (64, 32, 255),
                                      (20, 32, 97), (64, 4, 300), (128, 16, 700), (256, 16, 600), (300, 32, 700)])
@pytest.mark.parametrize("sweep", ["forward", "backward", "symmetric"])
def test_coop_emulation_matches_oracle(ps, tpp, n, sweep):
    A = W.poisson2d_matrix(int(math.ceil(math.sqrt(n))), eps=0.3)
    A = A[:n, :n].tocsc()
    A.sort_indices()
    x = np.random.default_rng(ps + n).uniform(-1, 1, n)
    ref = O.OracleL1GS(A, ps, isSymA=True, sweep=sweep, cache="packed")
    want = ref.ldiv(x)
    got = emulate(A, ps, tpp, sweep, ref.D, x, np.float64)
    if sweep == "forward":
        np.testing.assert_array_equal(got, want)
    else:
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-12 * np.abs(want).max())


def test_coop_emulation_fp32():
    A = W.poisson2d_matrix(20, eps=0.3).astype(np.float32)
    x = np.random.default_rng(1).uniform(-1, 1, A.shape[0]).astype(np.float32)
    for sweep in ("forward", "symmetric"):
        ref = O.OracleL1GS(A, 24, isSymA=True, sweep=sweep, cache="packed")
        got = emulate(A, 24, 16, sweep, ref.D, x, np.float32)
        want = ref.ldiv(x)
        if sweep == "forward":
            np.testing.assert_array_equal(got, want)
        else:
            np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5 * np.abs(want).max())


def test_coop_layout_covers_reference_packing():
    """Every strict-triangle slot of every partition maps to a distinct stream
    entry inside its group's stride (no collisions, no overrun)."""
    for ps, tpp in ((16, 4), (33, 16), (64, 32), (256, 32), (100, 16)):
        for lower, upper in ((True, False), (False, True), (True, True)):
            L = make_layout(ps, tpp, lower, upper, 8)
            seen = set()
            for k in range(2 * L["G"]):
                for li in range(ps):
                    for lj in range(ps):
                        if lj < li and lower:
                            p = lower_idx(L, k, li, lj)
                        elif lj > li and upper:
                            p = upper_idx(L, k, li, lj)
                        else:
                            continue
                        assert p not in seen
                        seen.add(p)
                        q = k // L["G"]
                        assert q * L["Lgp"] <= p < q * L["Lgp"] + L["Lg"]
            assert len(seen) == 2 * L["Lg"]
