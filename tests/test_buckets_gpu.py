"""Length buckets on the GPU: every task runs with its pair's bucket row of
kernel shapes (N <= 128, <= 512, longer), and with split = 1 a batch that
spans the buckets runs as one sub-batch per bucket side by side.  The
shapes change the schedule only, and every pair's search is independent of
the rest of its batch, so the results, the per-stage running bests and the
learned search's audit draws must equal those of one unsplit call with the
default shapes, bit for bit."""
from __future__ import annotations

import copy

import numpy as np
import pytest

import indialign_b200 as ia
from indialign_b200 import ranker, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mixed():
    rng = np.random.default_rng(71)
    pairs = []
    for L in (40, 70, 100, 128, 129, 200, 300, 512, 513, 700):
        pairs.append(W.make_pair(L, float(rng.uniform(0.5, 14)), rng, 0.05))
    return pairs


def _with(split, rows=None):
    t = ia.get_tuning()
    t = copy.deepcopy(t)
    t["split"] = split
    t["min_pairs"] = 2
    if rows:
        for b, r in rows.items():
            t["rows"][b].update(r)
    return t


@pytest.fixture
def table():
    before = ia.get_tuning()
    yield
    ia.set_tuning(before)


def _run(pairs, **kw):
    tr = np.zeros(len(pairs) * ia.TRACE_STAGES * 13)
    s, R, t = ia.search(pairs, stage_best=tr, **kw)
    return s, R, t, tr


def test_split_equals_one_call_plain(mixed, table):
    ia.set_tuning(_with(0))
    a = _run(mixed)
    ia.set_tuning(_with(1))
    b = _run(mixed)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_split_with_other_shapes_equals_one_call(mixed, table):
    """Other bank chunk sizes, item orders, chain chunks and trace placement
    per bucket change the schedule only, not the results."""
    ia.set_tuning(_with(0))
    a = _run(mixed)
    ia.set_tuning(_with(1, {0: dict(bank_chunk=64, bank_cutoff_major=0, chain_chunk=4, chain_smem_trace=1),
                            1: dict(bank_chunk=512, chain_chunk=32, chain_smem_trace=0),
                            2: dict(bank_chunk=128, bank_cutoff_major=0, chain_chunk=8)}))
    b = _run(mixed)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)


def test_split_equals_one_call_learned_with_audits(mixed, table):
    blob = ranker.default_weights()
    out = []
    for split in (0, 1):
        ia.set_tuning(_with(split))
        st = np.zeros(ia.RANK_STATS, np.int64)
        s, R, t = ia.search(mixed, ranker=blob, audit_rate=0.5, seed=3, rank_stats=st)
        out.append((s, R, t, st))
    for x, y in zip(out[0][:3], out[1][:3]):
        np.testing.assert_array_equal(x, y)
    a, b = out[0][3], out[1][3]
    bad = np.nonzero(a != b)[0]
    assert bad.size == 0, [(int(i) // 8, int(i) % 8, int(a[i]), int(b[i])) for i in bad]  # (kind, stat)
    assert a.reshape(ia.CAND_KINDS, -1)[:, 2].sum() > 0  # some lists were audited


def test_learned_stats_repeat(mixed, table):
    """Two identical unsplit learned calls give the same ranker statistics."""
    blob = ranker.default_weights()
    ia.set_tuning(_with(0))
    st = [np.zeros(ia.RANK_STATS, np.int64) for _ in range(2)]
    for k in range(2):
        ia.search(mixed, ranker=blob, audit_rate=0.5, seed=3, rank_stats=st[k])
    bad = np.nonzero(st[0] != st[1])[0]
    assert bad.size == 0, [(int(i) // 8, int(i) % 8, int(st[0][i]), int(st[1][i])) for i in bad]


def test_learned_results_do_not_depend_on_pair_order(mixed, table):
    """One unsplit learned call on the pairs in reverse order gives the same
    per-pair results (audit draws follow the pair's index, so the audit rate
    is 0 here) and the same ranker statistics."""
    blob = ranker.default_weights()
    ia.set_tuning(_with(0))
    rev = mixed[::-1]
    st = [np.zeros(ia.RANK_STATS, np.int64) for _ in range(2)]
    s0, R0, t0 = ia.search(mixed, ranker=blob, audit_rate=0.0, seed=3, rank_stats=st[0])
    s1, R1, t1 = ia.search(rev, ranker=blob, audit_rate=0.0, seed=3, rank_stats=st[1])
    np.testing.assert_array_equal(s0, s1[::-1])
    np.testing.assert_array_equal(R0, R1[::-1])
    bad = np.nonzero(st[0] != st[1])[0]
    assert bad.size == 0, [(int(i) // 8, int(i) % 8, int(st[0][i]), int(st[1][i])) for i in bad]


def test_split_device_entry(mixed, table):
    """The device-resident entry scatters each sub-batch's rows into the
    caller's output in batch order."""
    torch = pytest.importorskip("torch")
    import ctypes
    lens = [p.pred.shape[0] for p in mixed]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cat = lambda f, dt: torch.from_numpy(np.concatenate([np.asarray(f(p), dt).reshape(-1) for p in mixed])).cuda()
    dp, dn = cat(lambda p: p.pred, np.float64), cat(lambda p: p.native, np.float64)
    dv, dpv, dnv = (cat(lambda p: p.valid, np.uint8), cat(lambda p: p.pred_valid, np.uint8),
                    cat(lambda p: p.native_valid, np.uint8))
    ln = np.array([p.lnorm for p in mixed], np.float64)
    lib = ia.load()
    cfg = ia.default_config()
    outs = []
    for split in (0, 1):
        ia.set_tuning(_with(split))
        out = torch.full((len(mixed) * 13,), -5.0, dtype=torch.float64, device="cuda")
        opts = ia.BatchOptions()
        opts.device = torch.cuda.current_device()
        opts.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = lib.indialign_tmscore_search_device(
            len(mixed), off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), dp.data_ptr(), dn.data_ptr(),
            dv.data_ptr(), dpv.data_ptr(), dnv.data_ptr(), ln.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            ctypes.byref(cfg), ctypes.byref(opts), out.data_ptr())
        assert rc == 0, ia.last_error()
        torch.cuda.synchronize()
        outs.append(out.cpu().numpy())
    np.testing.assert_array_equal(outs[0], outs[1])
    s_h, _, _ = ia.search(mixed)
    np.testing.assert_array_equal(outs[1].reshape(-1, 13)[:, 0], s_h)
