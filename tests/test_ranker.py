"""CPU checks of the learned window ranker's host side and of its oracle:
the oracle's backward against FP64 finite differences, the window schedule
against the library's count, the training-pair assembly and the parameter
layout."""
from __future__ import annotations

import os
import re
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import ranker_oracle as ro  # noqa: E402

import indialign_b200 as ia  # noqa: E402
from indialign_b200 import ranker  # noqa: E402


def _blob(seed=0):
    rng = np.random.default_rng(seed)
    mean = rng.normal(0, 0.3, 16).astype(np.float32)
    std = rng.uniform(0.5, 2.0, 16).astype(np.float32)
    return ranker.init_blob(mean, std, seed)


def test_blob_layout_matches_header():
    hdr = open(os.path.join(ROOT, "include", "indialign_b200.h")).read()
    n = int(re.search(r"#define INDIALIGN_RANKER_FLOATS (\d+)", hdr).group(1))
    assert n == ia.RANKER_FLOATS == ro.SIZE == ranker.B3 + 1
    assert (ranker.W1, ranker.B1, ranker.W2, ranker.B2, ranker.W3) == (ro.W1, ro.B1, ro.W2, ro.B2, ro.W3)
    assert int(re.search(r"#define INDIALIGN_RANK_STATS (\d+)", hdr).group(1)) == ia.RANK_STATS


def test_oracle_backward_matches_finite_differences():
    """FP64 network (no BF16 rounding): analytic gradient of the loss equals
    central differences, so the oracle's backward is the true gradient."""
    rng = np.random.default_rng(3)
    blob = _blob(1).astype(np.float64)
    x = rng.normal(0, 1, (12, 16)).astype(np.float32)
    t = rng.uniform(0, 1, 12)
    y, _ = ro.mlp_forward(blob, x, emulate=False)
    _, dy = ro.loss(y, t, 0.7)
    g = ro.mlp_backward(blob, x, dy, emulate=False)

    def L(b):
        yy, _ = ro.mlp_forward(b, x, emulate=False)
        return ro.loss(yy, t, 0.7)[0]

    # the FP64 path still rounds weights to BF16 (as the device does), so
    # perturb along directions that keep BF16 weights exact: use biases, w3,
    # b3 directly, and check weight blocks through the chain rule on b.
    idx = list(range(ro.B1, ro.B1 + 6)) + list(range(ro.B2, ro.B2 + 6)) + list(range(ro.W3, ro.W3 + 6)) + [ro.B3]
    for i in idx:
        e = np.zeros_like(blob)
        h = 1e-5
        e[i] = h
        fd = (L(blob + e) - L(blob - e)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_oracle_weight_gradients_match_outer_products():
    """dW = input^T dz for both layers (weights enter only through BF16
    copies, so their gradient is checked against the bias gradients' rows)."""
    rng = np.random.default_rng(4)
    blob = _blob(2)
    x = rng.normal(0, 1, (10, 16)).astype(np.float32)
    dy = rng.normal(0, 1, 10)
    g = ro.mlp_backward(blob, x, dy, emulate=False)
    _, a = ro.mlp_forward(blob, x, emulate=False)
    gz2 = dy[:, None] * a["p"]["w3"][None, :] * ro.gelu_grad(a["z2"])
    np.testing.assert_allclose(g[ro.W2:ro.B2].reshape(128, 128), a["h1"].T @ gz2, rtol=1e-12, atol=1e-12)
    gz1 = (gz2 @ a["W2b"].T) * ro.gelu_grad(a["z1"])
    np.testing.assert_allclose(g[ro.W1:ro.B1].reshape(16, 128), a["xn"].T @ gz1, rtol=1e-12, atol=1e-12)


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.00390625, 1.01171875, 1.0078125 + 2 ** -9, -3.14159], np.float32)
    r = ro.bf16(v)
    # 1 + 2^-8 is a tie between 1 and 1 + 2^-7: even mantissa (1.0) wins
    assert r[0] == 1.0 and r[1] == 1.0
    assert r[2] == np.float32(1.015625)  # tie 1.01171875 -> even 1.015625
    assert abs(float(r[4]) + 3.140625) < 1e-7


@pytest.mark.parametrize("plen,nlen", [(3, 50), (4, 4), (40, 38), (64, 64), (170, 165), (300, 290),
                                       (380, 420), (999, 960)])
def test_candidate_schedules_match_library(plen, nlen):
    for kind in range(3):
        cs = ro.candidates(plen, nlen, kind)
        assert len(cs) == ia.candidate_count(plen, nlen, kind), kind
        for flen, ps, ns in cs:
            assert 3 <= flen <= min(plen, nlen) and ps + flen <= plen and ns + flen <= nlen
    # detailed searches: two slots, each room for the largest aligned set
    m = min(plen, nlen)
    room = max([len(ro.det_seeds(k)) for k in range(m + 1)])
    assert ia.candidate_count(plen, nlen, ia.CAND_DET) == 2 * room
    for flen, ps, ns in ro.det_seeds(m):
        assert flen >= 3 and ps == ns and ps + flen <= m
    # main seed bank: room for the largest seed table
    assert ia.candidate_count(plen, nlen, ia.CAND_MAIN) == 1024
    assert ia.candidate_count(plen, nlen, 5) == 0 and ia.candidate_count(-1, nlen, 0) == 0


def test_pair_rows_pairs_within_groups():
    rng = np.random.default_rng(0)
    group = np.repeat(np.arange(20), rng.integers(1, 30, 20))
    pairs = ranker.pair_rows(group, rng)
    assert (group[pairs[:, 0]] == group[pairs[:, 1]]).all()
    flat = pairs.reshape(-1)
    assert len(set(flat.tolist())) == flat.size
    counts = np.bincount(group)
    assert flat.size == int((counts // 2 * 2).sum())


def test_select_oracle_rules():
    s = np.array([0.1, 0.5, 0.5, 0.2, 0.9, 0.3, np.nan], np.float32)
    c, lst = ro.select(s, 3, 0.0, 0.0, 0, 0)
    assert c == 3 and lst == [1, 2, 4]          # ties keep the lower window
    c, lst = ro.select(s, 3, 0.5, 0.0, 0, 0)
    assert c == -1 and lst == [1, 2, 4]         # 0.9 - 0.5 < 0.5: fallback
    assert ro.select(s, 7, 0.0, 0.0, 0, 0)[0] == -1  # at most k windows
    assert ro.select(s, 3, 0.0, 1.0, 0, 0)[0] == -2  # audit everything
    draws = [ro.audit_draw(12345, p) for p in range(20000)]
    assert 0.015 < np.mean(np.array(draws) < 0.02) < 0.025


def test_learned_mode_rejects_missing_ranker():
    """Option checks happen before any device work (no GPU needed)."""
    import ctypes
    lib = ia.load()
    from indialign_b200 import abi, workloads
    pk = abi.PackedInputs(workloads.single(0))
    res = (abi.NativePairResult * 1)()
    opts = ia.BatchOptions()
    opts.device = -1
    opts.mode = ia.MODE_LEARNED
    cfg = ia.default_config()
    rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts), res)
    assert rc == -4 and "ranker" in ia.last_error()
    opts.mode = 7
    rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts), res)
    assert rc == -4 and "mode" in ia.last_error()
    blob = np.zeros(ia.RANKER_FLOATS, np.float32)
    for k in (-1, 33):  # top_k outside 1..32 (0 means the default 8)
        ia.learned_options(opts, blob, k, 0.02, 0.02, 0, None)
        rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts), res)
        assert rc == -4 and "top_k" in ia.last_error(), (k, rc, ia.last_error())
    opts2 = ia.BatchOptions()
    opts2.device = -1
    opts2.mode = ia.MODE_COLLECT  # no feature / label buffers
    rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts2), res)
    assert rc == -4 and "collect" in ia.last_error()


def test_checkpoint_roundtrip(tmp_path):
    rng = np.random.default_rng(0)
    blob = _blob(3)
    m = rng.normal(0, 1e-3, blob.size).astype(np.float32)
    v = rng.uniform(0, 1e-4, blob.size).astype(np.float32)
    p = str(tmp_path / "ck.npz")
    ranker.save_checkpoint(p, blob, m, v, 1234)
    b2, m2, v2, step = ranker.load_checkpoint(p)
    assert step == 1234
    for a, b in ((blob, b2), (m, m2), (v, v2)):
        assert np.array_equal(a, b)
    np.savez(str(tmp_path / "bad.npz"), magic=np.array("other"))
    with pytest.raises(ia.IndialignError):
        ranker.load_checkpoint(str(tmp_path / "bad.npz"))
