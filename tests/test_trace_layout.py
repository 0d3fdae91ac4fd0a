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
