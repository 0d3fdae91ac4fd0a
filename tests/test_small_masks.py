"""Small pairs (N = 3..24) under every mask-pattern class: all valid, none
valid, pred / native masks that differ, single valid residues, alternating
gaps, lnorm at and below the degenerate limit.  The oracle is checked
against the reference build on the CPU; the GPU library against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from indialign_b200 import abi, workloads as W


def _cases():
    out = []
    rng = np.random.default_rng(123)
    for N in (3, 4, 5, 7, 9, 12, 16, 24):
        x = W.make_trace(N, rng)
        nat = x + rng.normal(0, 1.0, (N, 3))
        nat = nat @ W.random_rotation(rng).T + rng.uniform(-20, 20, 3)
        one = np.ones(N, np.uint8)
        zero = np.zeros(N, np.uint8)
        alt = (np.arange(N) % 2 == 0).astype(np.uint8)
        single = zero.copy()
        single[N // 2] = 1
        rnd_p = (rng.uniform(size=N) > 0.3).astype(np.uint8)
        rnd_n = (rng.uniform(size=N) > 0.3).astype(np.uint8)
        for pv, nv in ((one, one), (zero, zero), (alt, one), (one, alt), (single, one), (rnd_p, rnd_n),
                       (alt, 1 - alt)):
            v = (pv & nv).astype(np.uint8)
            for lnorm in (float(N), 2.0, float(max(int(v.sum()), 1))):
                out.append(W.Pair(np.ascontiguousarray(x), np.ascontiguousarray(nat), v, pv.copy(), nv.copy(),
                                  lnorm))
    return out


def test_small_mask_cases_oracle_matches_reference(oracle, ref):
    pairs = _cases()
    rc, so, Ro, to = abi.run_batch(oracle, pairs, prefix="ora_")
    rc2, sr, Rr, tr = abi.run_batch(ref, pairs)
    assert rc == 0 and rc2 == 0
    np.testing.assert_allclose(so, sr, atol=1e-9)
    ok = np.abs(so - sr) <= 1e-9
    np.testing.assert_allclose(Ro[ok], Rr[ok], atol=1e-6)
    degen = np.array([p.lnorm <= 2.0 for p in pairs])
    assert np.all(sr[degen] == 0.0) and np.allclose(Rr[degen], np.eye(3).reshape(-1))


@pytest.mark.gpu
def test_small_mask_cases_gpu_vs_oracle(oracle):
    import indialign_b200 as ia
    pairs = _cases()
    s, R, t = ia.search(pairs)
    rc, so, _, _ = abi.run_batch(oracle, pairs, prefix="ora_")
    assert rc == 0
    assert np.all(s >= so - 1e-6), np.nonzero(s < so - 1e-6)
    # degenerate cases (lnorm <= 2 or no seed) return score 0 with the identity
    degen = np.array([p.lnorm <= 2.0 for p in pairs])
    assert np.all(s[degen] == 0.0)
    assert np.allclose(R[degen], np.eye(3).reshape(-1))
