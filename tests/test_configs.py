"""Non-default NativeConfig settings: no fragment seeds, no / two DP
refinement iterations, fewer cutoff iterations, rescue thresholds that force
every rescue pass, a low early-termination score.  The oracle is checked
against the reference build (CPU); the GPU library against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

from indialign_b200 import abi, workloads as W

CONFIGS = {
    "no_fragments": dict(use_fragment_search=0),
    "no_dp": dict(dp_iter=0),
    "dp2": dict(dp_iter=2),
    "max_iter5": dict(max_iter=5),
    "all_rescues": dict(rescue_score_1=0.95, rescue_score_2=0.9),
    "early_term": dict(early_term_score=0.4),
}


def _cfg(lib, prefix, **kw):
    c = abi.default_config(lib, prefix)
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def _pairs():
    return W.batch(8, 40, 90, seed=808, sigma_lo=1.0, sigma_hi=10.0)


@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_oracle_matches_reference(oracle, ref, name):
    pairs = _pairs()
    rc, so, _, _ = abi.run_batch(oracle, pairs, _cfg(oracle, "ora_", **CONFIGS[name]), prefix="ora_")
    rc2, sr, _, _ = abi.run_batch(ref, pairs, _cfg(ref, "indialign_", **CONFIGS[name]))
    assert rc == 0 and rc2 == 0
    np.testing.assert_allclose(so, sr, atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CONFIGS))
def test_config_gpu_vs_oracle(oracle, name):
    import indialign_b200 as ia
    pairs = _pairs()
    s, _, _ = ia.search(pairs, _cfg(ia.load(), "indialign_", **CONFIGS[name]))
    rc, so, _, _ = abi.run_batch(oracle, pairs, _cfg(oracle, "ora_", **CONFIGS[name]), prefix="ora_")
    assert rc == 0
    assert np.all(s >= so - 1e-6), (name, s - so)
