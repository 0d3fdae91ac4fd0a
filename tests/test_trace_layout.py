"""CPU replay of the NW trace layout of the chain kernels (k_chain.cu
nw_align_t): every store a lane makes lies inside the trace block
(nw_trace_words_for), and every cell the traceback can read is found at the
address the fill stored it, in a word stored after the cell was computed.

The replay follows the kernel's per-lane state machine: lane l owns rows
2l+1, 2l+2 of each 64-row stripe, row 0 of the lane computes column j0 at
each step, stripes repeat with period P = max(nlen+1, 64), and at every step
with step % 16 == 15 (and when a lane leaves a stripe) the lane stores its two
rows' words of step word step // 16."""
from __future__ import annotations

import pytest


def trace_words_for(np_, nn):
    P = max(nn + 1, 64)
    return ((np_ + 63) // 64) * 64 * ((P + 127) // 16)


def trace_word(i, w, P, G):
    k, ri = (i - 1) >> 6, (i - 1) & 63
    g = w + ((k * P + ri) >> 4) - ((k * P) >> 4)
    return (k * G + g) * 64 + ri


def replay(plen, nlen):
    P = max(nlen + 1, 64)
    G = (P + 127) // 16
    S = (plen + 63) >> 6
    last_lane = ((plen - 1) & 63) >> 1
    total = (S - 1) * P + 2 * last_lane + 1 + nlen + 1
    size = trace_words_for(plen, nlen)
    stored = {}  # address -> (stripe, row in stripe, step word, step of the store)

    def store(l, k, g0, gw, step):
        if 64 * k + 2 * l + 1 > plen:  # the lane has no row inside the matrix: no store
            return
        for r in (0, 1):
            a = (k * G + gw - g0) * 64 + 2 * l + r
            assert 0 <= a < size, (plen, nlen, l, k, gw)
            stored[a] = (k, 2 * l + r, gw, step)

    for l in range(32):
        k, j0, g0 = 0, 1 - 2 * l, 0
        for step in range(total):
            if j0 > P:
                if ((step - 1) & 15) != 15 and k < S:
                    store(l, k, g0, (step - 1) >> 4, step - 1)
                j0 -= P
                k += 1
                g0 = (k * P) >> 4
            if (step & 15) == 15 and k < S:
                store(l, k, g0, step >> 4, step)
            j0 += 1
        if ((total - 1) & 15) != 15 and k < S:
            store(l, k, g0, (total - 1) >> 4, total - 1)
    # every cell (i, j): its bits at step t = base(i) + j - 1, word t // 16
    for i in range(1, plen + 1):
        k, ri = (i - 1) >> 6, (i - 1) & 63
        base = k * P + ri
        for j in range(1, nlen + 1):
            t = base + j - 1
            wr = (t >> 4) - (base >> 4)
            a = trace_word(i, wr, P, G)
            assert a in stored, (plen, nlen, i, j)
            sk, sri, sgw, sstep = stored[a]
            assert (sk, sri, sgw) == (k, ri, t >> 4), (plen, nlen, i, j, stored[a])
            assert sstep >= t, (plen, nlen, i, j)  # the word holds the finished cell
    return len(stored), size


@pytest.mark.parametrize("plen,nlen", [(1, 1), (1, 5), (5, 1), (3, 3), (7, 40), (64, 64), (65, 130),
                                       (130, 65), (200, 151), (300, 287), (129, 63), (700, 300)])
def test_trace_layout_stores_in_bounds_and_reads_what_was_stored(plen, nlen):
    replay(plen, nlen)


def test_trace_block_size_of_the_fixed_scratch():
    """The allocation-free NW entry's fixed array is sized by the same
    formula for its 2048 x 2048 maximum."""
    assert trace_words_for(2048, 2048) == 32 * 64 * ((2049 + 127) // 16)


def replay_bits(plen, nlen):
    """Replay of the fill's direction-bit packing: each step a row's 2 bits
    enter the top of its word and the word moves down 2 bits (a funnel
    shift); full words are stored after their 16th step, partial words (a
    lane leaving a stripe, the last steps) shifted down by 32 - 2m first.
    Every cell's bits must be read back by the traceback's rule
    (word trace_word(i, w), bits 2 * ((base(i) + j - 1) % 16))."""
    P = max(nlen + 1, 64)
    G = (P + 127) // 16
    S = (plen + 63) >> 6
    last_lane = ((plen - 1) & 63) >> 1
    total = (S - 1) * P + 2 * last_lane + 1 + nlen + 1
    mem = {}

    def dir_of(i, j):
        return (i * 7 + j * 3) % 4

    def push(acc, d):
        return ((acc >> 2) | (d << 30)) & 0xFFFFFFFF

    for l in range(32):
        k, j0, g0 = 0, 1 - 2 * l, 0
        acc = [0, 0]

        def store(w, vals):
            if 64 * k + 2 * l + 1 > plen:  # no row inside the matrix: no store
                return
            for r in (0, 1):
                mem[(k * G + w - g0) * 64 + 2 * l + r] = vals[r]

        for step in range(total):
            if j0 > P:
                if ((step - 1) & 15) != 15 and k < S:
                    sh = 30 - 2 * ((step - 1) & 15)
                    store((step - 1) >> 4, [a >> sh for a in acc])
                j0 -= P
                k += 1
                g0 = (k * P) >> 4
            if j0 == 1:
                acc = [0, 0]
            for r in (0, 1):
                i, j = 64 * k + 2 * l + r + 1, j0 - r
                ok = k < S and i <= plen and 1 <= j <= nlen
                acc[r] = push(acc[r], dir_of(i, j) if ok else 3)
            if (step & 15) == 15:
                if k < S:
                    store(step >> 4, acc)
                acc = [0, 0]
            j0 += 1
        if ((total - 1) & 15) != 15 and k < S:
            sh = 30 - 2 * ((total - 1) & 15)
            store((total - 1) >> 4, [a >> sh for a in acc])
    for i in range(1, plen + 1):
        base = ((i - 1) >> 6) * P + ((i - 1) & 63)
        for j in range(1, nlen + 1):
            t = base + j - 1
            word = mem[trace_word(i, (t >> 4) - (base >> 4), P, G)]
            assert (word >> (2 * (t & 15))) & 3 == dir_of(i, j), (plen, nlen, i, j)


@pytest.mark.parametrize("plen,nlen", [(1, 1), (1, 5), (5, 1), (3, 3), (7, 40), (64, 64), (65, 130),
                                       (130, 65), (200, 151), (129, 63), (300, 287)])
def test_direction_bits_land_where_the_traceback_reads_them(plen, nlen):
    replay_bits(plen, nlen)


def _cell(diag_src, sc, up_enc, left_enc, gap):
    """The fill's cell rule (k_chain.cu nw_cell): with a gap penalty the sign
    of H carries "reached diagonally" and a gap out of such a cell pays it;
    ties prefer diag, then left, then up.  Returns (encoded H, dir)."""
    import math
    diag = diag_src + sc
    if gap == 0.0:
        up, left = up_enc, left_enc
    else:
        up = abs(up_enc) + (gap if math.copysign(1.0, up_enc) < 0 else 0.0)
        left = abs(left_enc) + (gap if math.copysign(1.0, left_enc) < 0 else 0.0)
    is_diag = diag >= up and diag >= left
    d = 0 if is_diag else (2 if left >= up else 1)
    nh = diag if is_diag else (left if left >= up else up)
    return (nh if (gap == 0.0 or not is_diag) else -nh), d


def replay_fill(S, gap):
    """The fill's wavefront schedule on an explicit matrix S (plen x nlen):
    lanes hold two rows of a 64-row stripe, H reaches the next lane by a
    shuffle of the previous step's row-1 value, lane 31 leaves the stripe's
    last row in the boundary array for lane 0 of the next stripe, a lane
    resets its rows on entering a stripe, and row 1's column-0 cell is
    replaced by the boundary +0.  Returns the (i, j) -> dir map of the matrix
    cells and the plain H of the last row."""
    plen, nlen = S.shape
    P = max(nlen + 1, 64)
    nS = (plen + 63) >> 6
    last_lane = ((plen - 1) & 63) >> 1
    total = (nS - 1) * P + 2 * last_lane + 1 + nlen + 1
    bH = [0.0] * (nlen + 1)
    st = [dict(k=0, j0=1 - 2 * l, i0=2 * l + 1, h0=0.0, h1=0.0, h0prev=0.0, up0prev=0.0, r0ok=False, r1ok=False,
               st31=False, ld0=False) for l in range(32)]
    dirs, last_row = {}, {}
    hv = (lambda h: h) if gap == 0.0 else abs
    for step in range(total):
        ups = [st[l - 1]["h1"] if l > 0 else st[0]["h1"] for l in range(32)]  # shuffle up by 1
        writes = []
        for l in range(32):
            c = st[l]
            up0 = ups[l]
            if c["j0"] > P:
                c["j0"] -= P
                c["k"] += 1
                c["i0"] += 64
            if c["j0"] == 1:
                c.update(h0=0.0, h1=0.0, h0prev=0.0, up0prev=0.0)
                c["r0ok"] = c["k"] < nS and c["i0"] <= plen
                c["r1ok"] = c["k"] < nS and c["i0"] + 1 <= plen
                c["st31"] = l == 31 and c["k"] + 1 < nS and c["r1ok"]
                c["ld0"] = c["k"] > 0 and c["r0ok"]
            j0, i0 = c["j0"], c["i0"]
            if l == 0:
                up0 = bH[j0] if (c["ld0"] and 1 <= j0 <= nlen) else 0.0
            a0, a1 = min(i0, plen) - 1, min(i0 + 1, plen) - 1
            jc = min((j0 - 1) % (1 << 32), nlen - 1)
            jc1 = min((j0 - 2) % (1 << 32), nlen - 1)
            n1, d1 = _cell(c["h0prev"], S[a1, jc1], c["h0"], c["h1"], gap)
            n0, d0 = _cell(c["up0prev"], S[a0, jc], up0, c["h0"], gap)
            if c["st31"] and 2 <= j0 <= nlen + 1:
                writes.append((j0 - 1, n1))
            for r, d, n, j in ((0, d0, n0, j0), (1, d1, n1, j0 - 1)):
                i = i0 + r
                if c["k"] < nS and i <= plen and 1 <= j <= nlen:
                    dirs[(i, j)] = d
                    if i == plen:
                        last_row[j] = hv(n)
            c["h0prev"] = hv(c["h0"])
            c["up0prev"] = hv(up0)
            c["h1"] = 0.0 if j0 == 1 else n1
            c["h0"] = n0
            c["j0"] += 1
        for j, v in writes:
            bH[j] = v
    return dirs, last_row


def direct_fill(S, gap):
    plen, nlen = S.shape
    H = [[0.0] * (nlen + 1) for _ in range(plen + 1)]
    dirs = {}
    hv = (lambda h: h) if gap == 0.0 else abs
    for i in range(1, plen + 1):
        for j in range(1, nlen + 1):
            H[i][j], dirs[(i, j)] = _cell(hv(H[i - 1][j - 1]), S[i - 1, j - 1], H[i - 1][j], H[i][j - 1], gap)
    return dirs, {j: hv(H[plen][j]) for j in range(1, nlen + 1)}


@pytest.mark.parametrize("plen,nlen,gap,seed", [(3, 3, 0.0, 1), (7, 40, 0.0, 2), (64, 64, 0.0, 3),
                                                (65, 70, 0.0, 4), (130, 65, -0.6, 5), (129, 63, -0.6, 6),
                                                (200, 90, 0.0, 7), (140, 140, -1.0, 8)])
def test_wavefront_fill_equals_row_by_row_fill(plen, nlen, gap, seed):
    """Same cells, same rule, evaluated in the kernel's wavefront order
    (with stripes, shuffles and the boundary row) and row by row: every
    direction and the last row's H agree.  Matrices with many ties (a few
    distinct values, some negative)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    S = rng.integers(-2, 5, size=(plen, nlen)).astype(np.float64) / 4.0
    d1, h1 = replay_fill(S, gap)
    d2, h2 = direct_fill(S, gap)
    assert d1 == d2
    assert h1 == h2


def replay_fill_rows(S, gap, R):
    """The wavefront fill with R rows per lane (stripes of 32R rows): row r
    of a lane computes column j0 - r, its up and diagonal inputs are row
    r-1's values from one and two steps earlier (row 0: the previous lane's
    last row, by a shuffle, or the boundary row), a row's column-0 cell is
    replaced by the boundary +0, and the period is max(nlen + R - 1, 32R).
    Returns the (i, j) -> dir map and the plain H of the last row."""
    plen, nlen = S.shape
    RS = 32 * R
    P = max(nlen + R - 1, RS)
    nS = (plen + RS - 1) // RS
    last_lane = ((plen - 1) % RS) // R
    total = (nS - 1) * P + R * last_lane + R - 1 + nlen
    bH = [0.0] * (nlen + 1)
    st = [dict(k=0, j0=1 - R * l, i0=R * l + 1, h=[0.0] * R, hp=[0.0] * R, up0prev=0.0, ok=[False] * R,
               st31=False, ld0=False) for l in range(32)]
    dirs, last_row = {}, {}
    hv = (lambda h: h) if gap == 0.0 else abs
    for step in range(total):
        ups = [st[l - 1]["h"][R - 1] if l > 0 else st[0]["h"][R - 1] for l in range(32)]
        writes = []
        for l in range(32):
            c = st[l]
            up0 = ups[l]
            if c["j0"] > P:
                c["j0"] -= P
                c["k"] += 1
                c["i0"] += RS
            if c["j0"] == 1:
                c["h"], c["hp"], c["up0prev"] = [0.0] * R, [0.0] * R, 0.0
                c["ok"] = [c["k"] < nS and c["i0"] + r <= plen for r in range(R)]
                c["st31"] = l == 31 and c["k"] + 1 < nS and c["ok"][R - 1]
                c["ld0"] = c["k"] > 0 and c["ok"][0]
            j0, i0 = c["j0"], c["i0"]
            if l == 0:
                up0 = bH[j0] if (c["ld0"] and 1 <= j0 <= nlen) else 0.0
            new = []
            for r in range(R):
                a = min(i0 + r, plen) - 1
                jc = min((j0 - r - 1) % (1 << 32), nlen - 1)
                if r == 0:
                    n, d = _cell(c["up0prev"], S[a, jc], up0, c["h"][0], gap)
                else:
                    n, d = _cell(c["hp"][r - 1], S[a, jc], c["h"][r - 1], c["h"][r], gap)
                new.append(n)
                i, j = i0 + r, j0 - r
                if c["k"] < nS and i <= plen and 1 <= j <= nlen:
                    dirs[(i, j)] = d
                    if i == plen:
                        last_row[j] = hv(n)
            if c["st31"] and 1 <= j0 - (R - 1) <= nlen:
                writes.append((j0 - (R - 1), new[R - 1]))
            c["up0prev"] = hv(up0)
            c["hp"] = [hv(v) for v in c["h"]]
            c["h"] = [0.0 if (r >= 1 and j0 == r) else new[r] for r in range(R)]
            c["j0"] += 1
        for j, v in writes:
            bH[j] = v
    return dirs, last_row


@pytest.mark.parametrize("R", [2, 4])
@pytest.mark.parametrize("plen,nlen,gap,seed", [(3, 3, 0.0, 1), (7, 40, 0.0, 2), (64, 64, 0.0, 3),
                                                (65, 70, 0.0, 4), (130, 65, -0.6, 5), (129, 63, -0.6, 6),
                                                (200, 90, 0.0, 7), (140, 140, -1.0, 8), (300, 20, 0.0, 9),
                                                (257, 130, -0.6, 10)])
def test_wavefront_fill_with_r_rows_per_lane(plen, nlen, gap, seed, R):
    import numpy as np
    rng = np.random.default_rng(seed)
    S = rng.integers(-2, 5, size=(plen, nlen)).astype(np.float64) / 4.0
    d1, h1 = replay_fill_rows(S, gap, R)
    d2, h2 = direct_fill(S, gap)
    assert d1 == d2
    assert h1 == h2
