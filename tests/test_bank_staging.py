"""The seed-bank kernel's in-place conversion of a staged FP64 point set to
centred FP32 (points_to_f32 in indialign_b200/csrc/k_bank.cu), replayed on
the CPU byte for byte: the shared region holds the bulk-copied doubles at
`lead` bytes (0 or 8: the copy starts at the source rounded down to 16
bytes); in round r every thread of the 128-thread CTA first reads point
128r + tid, then (after a barrier) writes its four floats (x, y, z, w) into
the residue-pair layout at the start of the region -- pair k = residues 2k,
2k+1 as {x_2k, x_2k+1, y_2k, y_2k+1} {z_2k, z_2k+1, w_2k, w_2k+1}, w = 1 for
a valid residue, an odd set ending with a zero point of w = 0.  No round may
overwrite a double that a later read still needs, and the region must hold
the converted set exactly."""
from __future__ import annotations

import numpy as np
import pytest

CTA = 128  # kBankChunk


def _region_bytes(nmax: int) -> int:
    """coord_bytes of k_bank: room for a 15-byte lead and the rounded-up tail."""
    return (nmax * 24 + 47) & ~15


def _float_slots(i: int):
    """Float indices of residue i's x, y, z, w in the pair layout."""
    b = (i >> 1) * 8 + (i & 1)
    return [b, b + 2, b + 4, b + 6]


def _replay(points: np.ndarray, lead: int, nmax: int, valid=None) -> np.ndarray:
    n = points.shape[0]
    region = bytearray(_region_bytes(nmax))
    region[lead:lead + 24 * n] = points.astype("<f8").tobytes()
    off = points.mean(0)  # points_mean: FP64 mean of all n points
    for base in range(0, n, CTA):
        idx = range(base, min(base + CTA, n))
        # reads of the round (before the barrier)
        vals = {i: np.frombuffer(bytes(region[lead + 24 * i:lead + 24 * i + 24]), "<f8") for i in idx}
        # writes of the round (after the barrier): its residues, and the zero
        # point after an odd set in the round that holds index n
        writers = list(idx) + ([n] if (n & 1) and base <= n < base + CTA else [])
        for i in writers:
            if i < n:
                w = 1.0 if valid is None or valid[i] != 0 else 0.0
                f = np.append(vals[i] - off, w).astype("<f4")
            else:
                f = np.zeros(4, "<f4")
            for slot, v in zip(_float_slots(i), f):
                region[4 * slot:4 * slot + 4] = v.tobytes()
                # every later read lies at or above lead + 24 * (base + CTA)
                assert 4 * slot + 4 <= lead + 24 * (base + CTA)
    pair_bytes = 32 * ((n + 1) // 2)
    assert lead + 24 * n <= len(region) and pair_bytes <= len(region)
    flat = np.frombuffer(bytes(region[:pair_bytes]), "<f4")
    if n & 1:  # the zero point after an odd set
        assert np.all(flat[_float_slots(n)] == 0)
    return np.array([flat[_float_slots(i)] for i in range(n)], dtype=np.float32)


@pytest.mark.parametrize("n", [1, 2, 3, 127, 128, 129, 255, 256, 257, 1000, 1500, 1501])
@pytest.mark.parametrize("lead", [0, 8])
def test_in_place_conversion_is_exact(n, lead):
    rng = np.random.default_rng(n + lead)
    pts = rng.standard_normal((n, 3)) * 30 + rng.uniform(-50, 50, 3)
    valid = (rng.uniform(size=n) > 0.1).astype(np.uint8) * rng.integers(1, 3, n).astype(np.uint8)
    got = _replay(pts, lead, nmax=n + 7, valid=valid)
    want = (pts - pts.mean(0)).astype(np.float32)
    np.testing.assert_array_equal(got[:, :3], want)
    np.testing.assert_array_equal(got[:, 3], (valid != 0).astype(np.float32))
