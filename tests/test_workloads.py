"""The synthetic workloads match their stated shapes: A-form stems (C1'
radius 8.9 A, rise 2.8 A/nt, twist 32.7 deg, 6-12 base pairs), 5.9 A loop
steps, Gaussian noise plus a rigid transform on the native, mask rates and
length / noise ranges."""
from __future__ import annotations

import math

import numpy as np

from indialign_b200 import workloads as W


def test_trace_geometry():
    rng = np.random.default_rng(0)
    x, segs = W.make_trace(300, rng, return_stems=True)
    assert x.shape == (300, 3)
    stem_step = math.sqrt((2 * W.RADIUS * math.sin(W.TWIST / 2)) ** 2 + W.RISE ** 2)
    n_stem = 0
    for a, b, is_stem in segs:
        d = np.linalg.norm(np.diff(x[a:b], axis=0), axis=1)
        if not is_stem:
            np.testing.assert_allclose(d, W.LOOP_STEP, rtol=1e-9)
            continue
        n_stem += 1
        full = b - a
        if full >= 2 * 6 + 4:  # a complete hairpin: 5' strand, 4-nt loop, 3' strand
            n_bp = (full - 4) // 2
            assert 6 <= n_bp <= 12
            np.testing.assert_allclose(d[:n_bp - 1], stem_step, rtol=1e-9)
            # residues j apart on a strand: chord of j twists at the radius, j rises
            s5 = x[a:a + n_bp]
            for j in (2, 3):
                want = math.sqrt((2 * W.RADIUS * math.sin(j * W.TWIST / 2)) ** 2 + (j * W.RISE) ** 2)
                np.testing.assert_allclose(np.linalg.norm(s5[j:] - s5[:-j], axis=1), want, rtol=1e-9)
    assert n_stem >= 5


def test_pair_noise_and_transform():
    p = W.single(0)[0]
    assert p.pred.shape == (64, 3) and p.lnorm == 64.0 and p.sigma == 2.0
    assert p.valid.all() and p.pred_valid.all() and p.native_valid.all()
    R, t = W._kabsch_np(p.pred, p.native)
    rmsd = np.sqrt(((p.pred @ R.T + t - p.native) ** 2).sum(1).mean())
    assert 2.4 < rmsd < 4.2  # ~ 2.0 * sqrt(3) minus what the fit absorbs


def test_batch_ranges_and_masks():
    pairs = W.batch(200, 40, 300, seed=3)
    L = np.array([p.pred.shape[0] for p in pairs])
    s = np.array([p.sigma for p in pairs])
    assert L.min() >= 40 and L.max() <= 300 and s.min() >= 0.5 and s.max() <= 14.0
    inv_p = 1 - np.concatenate([p.pred_valid for p in pairs]).mean()
    inv_n = 1 - np.concatenate([p.native_valid for p in pairs]).mean()
    assert 0.035 < inv_p < 0.065 and 0.035 < inv_n < 0.065
    for p in pairs[:20]:
        assert np.array_equal(p.valid, p.pred_valid & p.native_valid) and p.lnorm == p.pred.shape[0]


def test_hard_half_and_parallel_determinism():
    h = W.hard(40, seed=2)
    assert sum(p.hard for p in h) == 20
    L = np.array([p.pred.shape[0] for p in h])
    assert L.min() >= 30 and L.max() <= 1500
    a = W.parallel_batch(20, 40, 80, seed=9, procs=1)
    b = W.parallel_batch(20, 40, 80, seed=9, procs=2)
    assert all(np.array_equal(x.native, y.native) for x, y in zip(a, b))
