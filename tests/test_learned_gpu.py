"""GPU parity of the learned window ranker against its CPU oracle
(oracle/ranker_oracle.py), all through the library's C ABI:

* MLP forward, loss, backward (gradient check) and Adam on the BF16
  tensor-core kernels vs the oracle with the same BF16 rounding points;
* window features from COLLECT mode vs the FP64 restatement;
* top-k / margin / audit selection in LEARNED mode vs the oracle rule on the
  device's own predicted scores;
* the shipped trained ranker vs the plain search: mean and worst final
  TM-score change within the bars (>= -1e-4 mean, >= -1e-3 worst), far fewer
  windows refined, and a better hit rate than an untrained network.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ranker_oracle as ro  # noqa: E402

import indialign_b200 as ia  # noqa: E402
from indialign_b200 import abi, ranker, workloads as W  # noqa: E402

pytestmark = pytest.mark.gpu

# forward outputs: |gpu - oracle| <= 2e-3 + 1e-2 |y| (FP32 accumulation order
# and one-ulp BF16 flips of hidden activations)
Y_ATOL, Y_RTOL = 2e-3, 1e-2
# gradients: per block, ||gpu - oracle|| <= 2e-2 ||oracle||
G_REL = 2e-2


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _blob(seed):
    rng = np.random.default_rng(seed)
    mean = rng.normal(0, 0.3, 16).astype(np.float32)
    std = rng.uniform(0.5, 2.0, 16).astype(np.float32)
    b = ranker.init_blob(mean, std, seed)
    b[ro.B1:ro.W2] = rng.normal(0, 0.1, 128)
    b[ro.B2:ro.W3] = rng.normal(0, 0.1, 128)
    b[ro.B3] = 0.3
    return b


def _features(rng, n):
    return (rng.normal(0, 1, (n, 16)) * 0.8 + 0.1).astype(np.float32)


def test_mlp_forward_matches_oracle(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(0)
    blob = _blob(1)
    for n in (1, 15, 64, 1000, 8193):
        x = _features(rng, n)
        tr = ranker.Trainer(blob, batch=16)
        y = tr.forward(torch.tensor(x, device="cuda")).cpu().numpy()
        yo, _ = ro.mlp_forward(blob, x)
        np.testing.assert_allclose(y, yo, atol=Y_ATOL, rtol=Y_RTOL)


def test_mlp_loss_matches_oracle(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(2)
    n = 1001
    y = rng.uniform(0, 1, n).astype(np.float32)
    t = rng.uniform(0, 1, n).astype(np.float32)
    t[10] = t[11]  # tied labels: no ranking term
    lib = ia.load()
    dy = torch.empty(n, device="cuda")
    loss = torch.zeros(1, device="cuda")
    yt, tt = torch.tensor(y, device="cuda"), torch.tensor(t, device="cuda")
    assert lib.indialign_mlp_loss(yt.data_ptr(), tt.data_ptr(), n, ctypes.c_float(0.5), dy.data_ptr(),
                                  loss.data_ptr(), None) == 0
    torch.cuda.synchronize()
    Lo, dyo = ro.loss(y, t, 0.5)
    assert abs(float(loss.item()) - Lo) <= 1e-4 * abs(Lo)
    np.testing.assert_allclose(dy.cpu().numpy(), dyo, atol=1e-7, rtol=1e-4)


@pytest.mark.parametrize("n", [77, 256, 1000, 8192])
def test_mlp_backward_gradient_check(torch_cuda, n):
    """Gradients of the BF16 tensor-core backward vs the oracle (same
    rounding points, FP64 sums)."""
    torch = torch_cuda
    rng = np.random.default_rng(n)
    blob = _blob(3)
    x = _features(rng, n)
    t = rng.uniform(0, 1, n).astype(np.float32)
    tr = ranker.Trainer(blob, batch=n, lam=0.5)
    _, g = tr.gradients(torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda"))
    g = g.cpu().numpy().astype(np.float64)
    yo, _ = ro.mlp_forward(blob, x)
    # the device's dy comes from its own y; use the oracle's y for the
    # oracle side (y agrees to the forward tolerance)
    _, dyo = ro.loss(yo, t, 0.5)
    go = ro.mlp_backward(blob, x, dyo)
    assert np.all(g[:ro.W1] == 0)
    for name, a, b in (("W1", ro.W1, ro.B1), ("b1", ro.B1, ro.W2), ("W2", ro.W2, ro.B2),
                       ("b2", ro.B2, ro.W3), ("w3", ro.W3, ro.B3), ("b3", ro.B3, ro.SIZE)):
        err = np.linalg.norm(g[a:b] - go[a:b])
        ref = np.linalg.norm(go[a:b])
        assert err <= G_REL * ref + 1e-9, (name, err, ref)


def test_adam_step_matches_oracle(torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(5)
    blob = _blob(4)
    lib = ia.load()
    w = torch.tensor(blob, device="cuda")
    g = torch.tensor(rng.normal(0, 1e-2, blob.size).astype(np.float32), device="cuda")
    m = torch.tensor(rng.normal(0, 1e-3, blob.size).astype(np.float32), device="cuda")
    v = torch.tensor(rng.uniform(0, 1e-4, blob.size).astype(np.float32), device="cuda")
    wo, mo, vo = ro.adam(blob, g.cpu().numpy(), m.cpu().numpy(), v.cpu().numpy(), 3, 1e-3)
    f = ctypes.c_float
    assert lib.indialign_mlp_adam(w.data_ptr(), g.data_ptr(), m.data_ptr(), v.data_ptr(), 3, f(1e-3),
                                  f(0.9), f(0.999), f(1e-8), None) == 0
    torch.cuda.synchronize()
    np.testing.assert_allclose(w.cpu().numpy(), wo, rtol=1e-5, atol=1e-7)
    np.testing.assert_allclose(m.cpu().numpy(), mo, rtol=1e-5, atol=1e-9)
    np.testing.assert_allclose(v.cpu().numpy(), vo, rtol=1e-5, atol=1e-12)
    assert np.array_equal(w.cpu().numpy()[:ro.W1], blob[:ro.W1])


def test_training_reduces_loss(torch_cuda):
    """A few hundred Adam steps of the device trainer fit a smooth target."""
    torch = torch_cuda
    rng = np.random.default_rng(6)
    n = 4096
    x = _features(rng, n)
    t = (0.3 + 0.2 * np.tanh(x[:, 0] - 0.5 * x[:, 5]) + 0.05 * x[:, 3]).astype(np.float32)
    tr = ranker.Trainer(ranker.init_blob(x.mean(0), x.std(0), 0), batch=n, lr=3e-3, lam=0.2)
    X, T = torch.tensor(x, device="cuda"), torch.tensor(t, device="cuda")

    def mse():
        return float(((tr.forward(X) - T) ** 2).mean().item())

    first = mse()
    for _ in range(300):
        tr.step(X, T)
    assert mse() < 0.05 * first


def _compact(p, ss):
    pv, nv = p.pred_valid.astype(bool), p.native_valid.astype(bool)
    return p.pred[pv], p.native[nv], "".join(np.array(list(ss[0]))[pv]), "".join(np.array(list(ss[1]))[nv])


def _ss(oracle, xyz, v):
    N = xyz.shape[0]
    buf = ctypes.create_string_buffer(N)
    oracle.ora_assign_ss(np.ascontiguousarray(xyz).ctypes.data_as(ctypes.c_void_p),
                         np.ascontiguousarray(v, np.uint8).ctypes.data_as(ctypes.c_void_p), N, buf)
    return buf.raw[:N].decode()


def _d0(L):
    L = max(L, 1.0)
    d0 = 0.3 if L <= 11 else 0.4 if L <= 15 else 0.5 if L <= 19 else 0.6 if L <= 23 else 0.7
    if L >= 30:
        d0 = 0.6 * np.sqrt(L - 0.5) - 2.5
    return max(d0, 0.3)


def test_candidate_features_match_oracle(oracle):
    """COLLECT-mode features of all three candidate kinds vs the FP64
    restatement (running best entering each pass from the stage trace)."""
    oracle.ora_assign_ss.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_char_p]
    pairs = [p for p in W.batch(24, 40, 160, seed=11, sigma_lo=6.0, sigma_hi=14.0)]
    stage_best = np.zeros(len(pairs) * ia.TRACE_STAGES * 13)
    ia.search(pairs, stage_best=stage_best)
    (_, _, _), feat, label, off = ia.collect_windows(pairs)
    sb = stage_best.reshape(len(pairs), ia.TRACE_STAGES, 13)
    checked = np.zeros(3, int)
    rng = np.random.default_rng(0)
    for i, p in enumerate(pairs):
        ss = (_ss(oracle, p.pred, p.pred_valid), _ss(oracle, p.native, p.native_valid))
        Pc, Qc, ssp, ssn = _compact(p, ss)
        for kind in range(3):  # detailed-search seeds live on device-only alignments
            lab = label[off[kind, i]:off[kind, i + 1]]
            if lab.size == 0 or np.isnan(lab).all():
                continue
            cs = ro.candidates(Pc.shape[0], Qc.shape[0], kind)
            assert len(cs) == lab.size
            best = sb[i, (2, 3, 4)[kind], 0]  # running best entering the pass
            for w in rng.choice(len(cs), size=min(10, len(cs)), replace=False):
                fo = ro.window_features(Pc, Qc, ssp, ssn, _d0(p.lnorm), p.lnorm, best, cs[w], kind)
                fg = feat[off[kind, i] + w].astype(np.float64)
                np.testing.assert_allclose(fg, fo, rtol=1e-5, atol=2e-6, err_msg=f"pair {i} kind {kind} cand {w}")
                checked[kind] += 1
    assert (checked >= 20).all(), checked


def _learned_run(pairs, blob, k=8, margin=0.02, audit=0.02, seed=0, outputs=True, min_len=-1, mask=0):
    lib = ia.load()
    pk = abi.PackedInputs(pairs)
    res = (abi.NativePairResult * pk.n)()
    opts = ia.BatchOptions()
    opts.device = -1
    stats = np.zeros(ia.RANK_STATS, np.int64)
    ia.learned_options(opts, blob, k, margin, audit, seed, stats, rank_mask=mask, rank_min_len=min_len)
    off = ia.candidate_offsets(pairs)
    C = int(off[-1, -1])
    score = np.zeros(max(1, C), np.float32)
    sel = np.zeros((6 * len(pairs), 33), np.int32)
    if outputs:
        opts.win_score = score.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
        opts.win_cap = C
        opts.win_select = sel.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
    cfg = ia.default_config()
    rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts), res)
    assert rc == 0, ia.last_error()
    return abi.results_to_numpy(res, pk.n), stats.reshape(ia.CAND_KINDS, -1), score, sel, off


def _lists(kind, n, off):
    """(selection row, pair, candidate range) of every list of a kind."""
    if kind < 3:
        return [(kind * n + i, i, off[kind, i], off[kind, i + 1]) for i in range(n)]
    if kind == 4:
        return [(5 * n + i, i, off[kind, i], off[kind, i + 1]) for i in range(n)]
    out = []
    for i in range(n):
        a, b = off[kind, i], off[kind, i + 1]
        h = (b - a) // 2
        out += [(3 * n + 2 * i, i, a, a + h), (3 * n + 2 * i + 1, i, a + h, b)]
    return out


def test_selection_matches_oracle():
    pairs = W.batch(48, 40, 200, seed=12, sigma_lo=5.0, sigma_hi=14.0)
    blob = _blob(7)
    for k, margin, audit, seed in ((8, 0.0, 0.0, 0), (8, 0.02, 0.3, 99), (3, 1e9, 0.0, 1), (32, 0.0, 0.0, 2)):
        (sc, _, _), stats, score, sel, off = _learned_run(pairs, blob, k, margin, audit, seed,
                                                          mask=(ia.RANK_LOCAL | ia.RANK_THREAD | ia.RANK_DENSE |
                                                                ia.RANK_DET_SS | ia.RANK_MAIN))
        for kind in range(ia.CAND_KINDS):
            gated = 0
            for r, i, a, b in _lists(kind, len(pairs), off):
                row = sel[r]
                if row[0] == -1 and (row[1:] == -1).all():
                    continue  # pass not run for this list (or at most k candidates)
                gated += 1
                s = score[a:b]
                if kind >= 3:  # this search's seeds only: scores up to its seed count
                    fin = np.isfinite(s)
                    s = s[:int(np.argmin(fin)) if not fin.all() else s.size]
                c, lst = ro.select(s, k, margin, audit, seed, i)
                assert row[0] == c, (kind, i, k, margin, audit)
                assert list(row[1:1 + k]) == lst
            st = stats[kind]
            assert st[0] >= gated
            assert st[1] + st[2] + st[3] + st[7] == st[0]
        assert stats[:, 0].sum() > 0


@pytest.fixture(scope="module")
def shipped():
    if not os.path.exists(ranker.WEIGHTS_PATH):
        pytest.skip("trained weights not shipped")
    return ranker.default_weights()


def test_learned_vs_plain_delta_tm(shipped):
    """The trained ranker on held-out pairs (L 40-1000, sigma 0.5-14, 5 %
    invalid): final TM-scores vs the plain search within the bars, and the
    rescue passes refine a small fraction of their candidates."""
    pairs = W.batch(256, 40, 1000, seed=4242)
    plain, _, _ = ia.search(pairs)
    (lsc, _, _), stats, _, _, _ = _learned_run(pairs, shipped, outputs=False, min_len=0)
    d = lsc - plain
    assert d.mean() >= -1e-4, d.mean()
    assert d.min() >= -1e-3, d.min()
    assert stats[:, 0].sum() > 0
    assert stats[:, 5].sum() < 0.5 * stats[:, 4].sum(), stats  # refined vs candidates


def test_trained_ranker_beats_untrained(shipped):
    """What the trained network gains: with the margin fallback and the
    audit off, its top-8 candidates contain the best refined score far more
    often than an untrained network's."""
    pairs = W.batch(96, 40, 300, seed=777, sigma_lo=6.0, sigma_hi=14.0)
    (_, _, _), _, label, off = ia.collect_windows(pairs)

    def hit_rate(blob):
        (_, _, _), _, score, sel, _ = _learned_run(pairs, blob, 8, -1.0, 0.0, 0)
        hits = tot = 0
        for kind in range(3):  # rescue passes: the same candidates in both runs
            for r, i, a, b in _lists(kind, len(pairs), off):
                if sel[r, 0] != 8:
                    continue
                lab = label[a:b]
                if np.isnan(lab).any():
                    continue
                tot += 1
                hits += lab[sel[r, 1:9]].max() >= lab.max() - 1e-3
        return hits / max(tot, 1), tot

    h_tr, n_tr = hit_rate(shipped)
    untrained = ranker.init_blob(shipped[:16], shipped[16:32], 123)
    h_un, _ = hit_rate(untrained)
    assert n_tr >= 10
    assert h_tr >= h_un + 0.15, (h_tr, h_un)


def test_learned_mode_with_full_fallback_is_the_plain_search():
    """With every list falling back (margin above any score gap) or no list
    ranked, the learned search refines every candidate in the plain order:
    results are bit-identical to the plain search."""
    pairs = W.batch(32, 40, 200, seed=21, sigma_lo=4.0, sigma_hi=14.0)
    s0, R0, t0 = ia.search(pairs)
    blob = _blob(9)
    for mask, margin in ((0, 1e9), (1 << 10, 0.0)):  # 1 << 10 names no list kind
        lib = ia.load()
        pk = abi.PackedInputs(pairs)
        res = (abi.NativePairResult * pk.n)()
        opts = ia.BatchOptions()
        opts.device = -1
        stats = np.zeros(ia.RANK_STATS, np.int64)
        ia.learned_options(opts, blob, 8, margin, 0.0, 0, stats, mask)
        cfg = ia.default_config()
        assert lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts), res) == 0
        s, R, t = abi.results_to_numpy(res, pk.n)
        np.testing.assert_array_equal(s, s0)
        np.testing.assert_array_equal(R, R0)
        np.testing.assert_array_equal(t, t0)
        st = stats.reshape(ia.CAND_KINDS, -1)
        if mask == 0:
            assert st[:, 0].sum() > 0 and st[:, 3].sum() == 0  # ranked, never pruned
        else:
            assert st.sum() == 0


def test_trainer_checkpoint_restores_state(torch_cuda, tmp_path):
    torch = torch_cuda
    rng = np.random.default_rng(8)
    x = torch.tensor(_features(rng, 512), device="cuda")
    t = torch.tensor(rng.uniform(0, 1, 512).astype(np.float32), device="cuda")
    a = ranker.Trainer(_blob(5), batch=512)
    for _ in range(5):
        a.step(x, t)
    path = str(tmp_path / "ck.npz")
    a.checkpoint(path)
    b = ranker.Trainer(_blob(6), batch=512)
    b.restore(path)
    a.step(x, t)
    b.step(x, t)
    assert b.steps == a.steps == 6
    np.testing.assert_array_equal(a.numpy_blob(), b.numpy_blob())


def test_main_seed_features_match_oracle(oracle):
    """COLLECT-mode features of the main seed bank's seeds (fragment windows
    and anchors, from the oracle's own seed builder) vs the FP64
    restatement."""
    u8p = ctypes.POINTER(ctypes.c_uint8)
    dp = ctypes.POINTER(ctypes.c_double)
    oracle.ora_all_seeds.argtypes = [dp, dp, u8p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                     u8p, ctypes.c_int]
    oracle.ora_all_seeds.restype = ctypes.c_int
    oracle.ora_seed_masks.argtypes = [ctypes.c_int, u8p, ctypes.c_int, ctypes.c_int, u8p, ctypes.c_int]
    oracle.ora_seed_masks.restype = ctypes.c_int
    oracle.ora_d0.argtypes = [ctypes.c_double, dp, dp, dp]
    pairs = W.batch(12, 40, 160, seed=13)
    (_, _, _), feat, label, off = ia.collect_windows(pairs)
    rng = np.random.default_rng(1)
    checked = 0
    for i, p in enumerate(pairs):
        N = p.pred.shape[0]
        P, Q = np.ascontiguousarray(p.pred), np.ascontiguousarray(p.native)
        v = np.ascontiguousarray(p.valid, np.uint8)
        d0, d0s, sd8 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        oracle.ora_d0(p.lnorm, ctypes.byref(d0), ctypes.byref(d0s), ctypes.byref(sd8))
        masks = np.zeros((1024, N), np.uint8)
        K = oracle.ora_all_seeds(P.ctypes.data_as(dp), Q.ctypes.data_as(dp), v.ctypes.data_as(u8p), N,
                                 d0s.value, d0.value, 1, masks.ctypes.data_as(u8p), 1024)
        lab = label[off[4, i]:off[4, i + 1]]
        assert int(np.isfinite(lab).sum()) == K, (i, K)
        for w in rng.choice(K, size=min(12, K), replace=False):
            fo = ro.main_seed_features(P, Q, v, masks[w], w >= _frag_count(oracle, N, v), d0.value, d0s.value,
                                       p.lnorm)
            np.testing.assert_allclose(feat[off[4, i] + w].astype(np.float64), fo, rtol=1e-5, atol=2e-6,
                                       err_msg=f"pair {i} seed {w}")
            checked += 1
    assert checked >= 60


def _frag_count(oracle, N, v):
    """Number of fragment-window seeds (the anchors follow them)."""
    buf = np.zeros((1024, N), np.uint8)
    u8p = ctypes.POINTER(ctypes.c_uint8)
    return oracle.ora_seed_masks(N, v.ctypes.data_as(u8p), 1, 50, buf.ctypes.data_as(u8p), 1024)
