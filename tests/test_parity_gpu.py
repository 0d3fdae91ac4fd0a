"""Parity of the CUDA search with the reference, through the C ABI.

Bar (per pair): final TM-score >= reference - 1e-6 after the FP64 same-index
rescoring the search ends with; |dTM| and the rotation error against the
reference are reported.  Checked on the golden fixtures (reference outputs
committed under tests/golden/) and on fresh seeded inputs against the oracle.
"""
import ctypes
import threading

import numpy as np
import pytest

from conftest import GoldenPairs, rot_err_deg
import indialign_b200 as ia
from indialign_b200 import abi, workloads as W

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _report(tag, s, ref):
    d = s - ref
    print(f"[{tag}] n={len(s)} min dTM={d.min():.3e} max|dTM|={np.abs(d).max():.3e}")


def test_golden_final_scores(golden):
    s, R, t = ia.search(golden.pairs)
    _report(golden.name, s, golden.score)
    assert np.all(s >= golden.score - TOL), np.nonzero(s < golden.score - TOL)


def test_golden_stage_trace(golden):
    n = len(golden.pairs)
    tr = np.zeros(n * ia.TRACE_STAGES * 13)
    ia.search(golden.pairs, stage_best=tr)
    tr = tr.reshape(n, ia.TRACE_STAGES, 13)
    ref = golden.trace
    bad = []
    for k in range(n):
        for st in range(ia.TRACE_STAGES):
            if ref[k, st, 0] > -1e30 and abs(tr[k, st, 0] - ref[k, st, 0]) > TOL:
                bad.append((k, st, tr[k, st, 0], ref[k, st, 0]))
    assert not bad, bad[:10]


def test_fresh_pairs_vs_oracle(oracle):
    pairs = W.batch(24, 40, 140, seed=4242)
    s, R, t = ia.search(pairs)
    rc, so, Ro, to = abi.run_batch(oracle, pairs, prefix="ora_")
    assert rc == 0
    _report("fresh", s, so)
    assert np.all(s >= so - TOL)
    agree = np.abs(s - so) <= TOL
    assert rot_err_deg(R[agree], Ro[agree]).max() < 1e-3


def test_rotation_is_proper_and_score_is_rescored():
    pairs = W.batch(8, 40, 120, seed=77)
    s, R, t = ia.search(pairs)
    for k, p in enumerate(pairs):
        M = R[k].reshape(3, 3)
        assert np.allclose(M @ M.T, np.eye(3), atol=1e-9)
        assert abs(np.linalg.det(M) - 1) < 1e-9
        # aligned_d = sum_k p_k R[3k+d] + t_d  ->  x @ M + t
        moved = p.pred @ M + t[k]
        L = p.pred.shape[0]
        d0 = max(0.6 * np.sqrt(L - 0.5) - 2.5, 0.3) if L >= 30 else None
        if d0 is None:
            continue
        d2 = np.sum((moved - p.native) ** 2, 1)
        tm = np.sum((1 / (1 + d2 / d0 ** 2))[p.valid != 0]) / max(p.lnorm, 1)
        assert abs(tm - s[k]) < 1e-9


def test_identity_pair_scores_one():
    x = W.make_trace(60, np.random.default_rng(3))
    one = np.ones(60, np.uint8)
    s, R, t = ia.search([W.Pair(x, x.copy(), one, one, one, 60.0)])
    assert s[0] > 0.999999


def test_device_entry_matches_host_entry():
    torch = pytest.importorskip("torch")
    pairs = W.batch(6, 40, 100, seed=31)
    s_h, R_h, t_h = ia.search(pairs)
    lens = [p.pred.shape[0] for p in pairs]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cat = lambda f, dt: torch.from_numpy(np.concatenate([np.asarray(f(p), dt).reshape(-1) for p in pairs])).cuda()
    dp, dn = cat(lambda p: p.pred, np.float64), cat(lambda p: p.native, np.float64)
    dv, dpv, dnv = (cat(lambda p: p.valid, np.uint8), cat(lambda p: p.pred_valid, np.uint8),
                    cat(lambda p: p.native_valid, np.uint8))
    ln = np.array([p.lnorm for p in pairs], np.float64)
    out = torch.zeros(len(pairs) * 13, dtype=torch.float64, device="cuda")
    lib = ia.load()
    cfg = ia.default_config()
    opts = ia.BatchOptions()
    opts.device = torch.cuda.current_device()
    torch.cuda.synchronize()
    rc = lib.indialign_tmscore_search_device(
        len(pairs), off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), dp.data_ptr(), dn.data_ptr(),
        dv.data_ptr(), dpv.data_ptr(), dnv.data_ptr(),
        ln.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(cfg), ctypes.byref(opts),
        out.data_ptr())
    assert rc == 0, ia.last_error()
    o = out.cpu().numpy().reshape(-1, 13)
    np.testing.assert_array_equal(o[:, 0], s_h)
    np.testing.assert_array_equal(o[:, 1:10], R_h)


def test_concurrent_calls_are_independent():
    a = W.batch(4, 40, 90, seed=5)
    b = W.batch(4, 40, 90, seed=6)
    ref_a, ref_b = ia.search(a)[0], ia.search(b)[0]
    out = {}

    def run(name, pairs):
        out[name] = ia.search(pairs)[0]

    th = [threading.Thread(target=run, args=(f"a{i}", a)) for i in range(2)] + \
         [threading.Thread(target=run, args=(f"b{i}", b)) for i in range(2)]
    for x in th:
        x.start()
    for x in th:
        x.join()
    for i in range(2):
        np.testing.assert_array_equal(out[f"a{i}"], ref_a)
        np.testing.assert_array_equal(out[f"b{i}"], ref_b)


def test_injected_failure_leaves_context_usable():
    lib = ia.load()
    lib.indialign_inject_failure(1)
    with pytest.raises(ia.IndialignError, match="rc=-6"):
        ia.search(W.single(0))
    s, _, _ = ia.search(W.single(0))
    assert s[0] > 0.3


def test_newton_reciprocal_within_one_ulp():
    """rcp_nr (float seed + 2 Newton steps) against the correctly rounded 1/x
    over the ranges the search feeds it (1 + d2/d0^2 and Jacobi pivots)."""
    rng = np.random.default_rng(0)
    x = np.concatenate([1.0 + rng.exponential(50.0, 20000), 10 ** rng.uniform(-14, 25, 20000),
                        -(10 ** rng.uniform(-14, 25, 5000))])
    y = np.zeros_like(x)
    lib = ia.load()
    lib.indialign_selftest_rcp.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                           ctypes.POINTER(ctypes.c_double)]
    assert lib.indialign_selftest_rcp(len(x), x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                      y.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 0
    exact = 1.0 / x
    ulp = np.abs(y - exact) / np.spacing(np.abs(exact))
    assert ulp.max() <= 1.0, ulp.max()


def test_nw_explicit_bit_exact_vs_reference():
    """Given an identical FP64 score matrix, the device NW (fill + traceback)
    returns exactly the reference's alignment, ties included."""
    import os
    torch = pytest.importorskip("torch")
    lib = ia.load()
    lib.indialign_nw_align.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    lib.indialign_nw_align.restype = ctypes.c_int
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_nw.npz"))
    k = 0
    while f"q{k}" in z:
        m = torch.from_numpy(np.ascontiguousarray(z[f"q{k}"].astype(np.float64) / 4096.0)).cuda()
        npr, nn = m.shape
        ap = torch.zeros(min(npr, nn), dtype=torch.int32, device="cuda")
        an = torch.zeros_like(ap)
        na = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = lib.indialign_nw_align(m.data_ptr(), npr, nn, float(z[f"g{k}"][0]), ap.data_ptr(),
                                    an.data_ptr(), na.data_ptr(), None)
        assert rc == 0, ia.last_error()
        n = int(na.item())
        np.testing.assert_array_equal(ap[:n].cpu().numpy(), z[f"ap{k}"], err_msg=f"case {k}")
        np.testing.assert_array_equal(an[:n].cpu().numpy(), z[f"an{k}"], err_msg=f"case {k}")
        k += 1
    assert k >= 90


def test_padded_tensor_entry_matches_host_entry():
    """The (B, N, 3) padded-tensor entry gives the same results as the host
    batch entry on the same pairs (padding rows hold garbage on purpose)."""
    import torch
    pairs = W.batch(6, 40, 120, seed=99)
    s_h, R_h, t_h = ia.search(pairs)
    N = max(p.pred.shape[0] for p in pairs) + 7
    B = len(pairs)
    rng = np.random.default_rng(0)
    P = rng.normal(0, 50, (B, N, 3))
    Q = rng.normal(0, 50, (B, N, 3))
    V, PV, NV = (np.ones((B, N), np.uint8) for _ in range(3))
    lens = np.zeros(B, np.int32)
    for i, p in enumerate(pairs):
        L = p.pred.shape[0]
        lens[i] = L
        P[i, :L], Q[i, :L] = p.pred, p.native
        V[i, :L], PV[i, :L], NV[i, :L] = p.valid, p.pred_valid, p.native_valid
    t = lambda a: torch.tensor(a, device="cuda")
    s, R, tt = ia.search_tensors(t(P), t(Q), t(V), t(PV), t(NV), lengths=lens,
                                 lnorm=np.array([p.lnorm for p in pairs]))
    np.testing.assert_array_equal(s.cpu().numpy(), s_h)
    np.testing.assert_array_equal(R.cpu().numpy(), R_h)
    np.testing.assert_array_equal(tt.cpu().numpy(), t_h)


def test_search_multi_matches_single_call():
    """Sharded over the visible devices (listed twice to exercise concurrent
    contexts on one GPU): same results as one batched call."""
    import torch
    pairs = W.batch(10, 40, 150, seed=31)
    s0, R0, t0 = ia.search(pairs)
    devs = list(range(torch.cuda.device_count())) * 2
    s, R, t = ia.search_multi(pairs, devs)
    np.testing.assert_array_equal(s, s0)
    np.testing.assert_array_equal(R, R0)
    np.testing.assert_array_equal(t, t0)


def test_profile_env_prints_every_stage(capfd, monkeypatch):
    """INDIALIGN_PROFILE prints the per-stage device times under the
    reference's stage names, tagged with INDIALIGN_PROFILE_TAG."""
    monkeypatch.setenv("INDIALIGN_PROFILE", "1")
    monkeypatch.setenv("INDIALIGN_PROFILE_TAG", "[t]")
    ia.search(W.batch(3, 40, 80, seed=5))
    err = capfd.readouterr().err
    names = ["seed_build", "seed_bank", "ss", "gapless_threading", "local_fragment", "threading_dp",
             "dense_local_fragment", "topk_seed", "dp_refine", "offset_dp", "weighted_refine", "total"]
    for nm in names:
        assert f"[indialign][t] pairs=3 stage={nm} ms=" in err, nm


def _walk_chain(N, rng):
    """Persistent random walk of 5.9 A steps (a crude C1' chain)."""
    steps = np.empty((N, 3))
    d = rng.normal(size=3)
    for i in range(N):
        d = d / np.linalg.norm(d) + 0.3 * rng.normal(size=3)
        steps[i] = d / np.linalg.norm(d) * (5.9 + 0.5 * rng.normal())
    x = np.cumsum(steps, 0)
    return x - x.mean(0)


@pytest.mark.parametrize("N,sigma,floor", [(50, 1.0, 0.5), (200, 3.0, 0.2), (6000, 2.0, 0.3),
                                           (8192, 2.0, 0.3)])
def test_long_chains_like_the_reference_smoke_cases(N, sigma, floor):
    """The reference C path's own smoke cases (random-walk chains, rotated,
    Gaussian noise; rc 0 and a score floor), including N = 6000 and 8192,
    which run the kernels' global-memory variants (point sets and NW rows
    beyond shared memory)."""
    rng = np.random.default_rng(N)
    nat = _walk_chain(N, rng)
    pred = nat @ W.random_rotation(rng).T + rng.normal(0, sigma, (N, 3))
    ones = np.ones(N, np.uint8)
    p = W.Pair(np.ascontiguousarray(pred), np.ascontiguousarray(nat), ones, ones, ones, float(N), sigma, False)
    s, R, t = ia.search([p])
    assert s[0] > floor, s
    # the returned transform reproduces the returned same-index score
    moved = pred @ R[0].reshape(3, 3) + t[0]
    d2 = ((moved - nat) ** 2).sum(1)
    L = float(N)
    d0 = max(0.6 * np.sqrt(L - 0.5) - 2.5, 0.3)
    assert abs((1.0 / (1.0 + d2 / d0 ** 2)).sum() / L - s[0]) < 1e-9


def test_identity_long_chain_scores_one():
    rng = np.random.default_rng(3)
    nat = _walk_chain(100, rng)
    ones = np.ones(100, np.uint8)
    s, _, _ = ia.search([W.Pair(nat.copy(), nat, ones, ones, ones, 100.0, 0.0, False)])
    assert s[0] > 0.95
