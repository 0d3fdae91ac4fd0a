"""The seed-bank kernel's in-place conversion of a staged FP64 point set to
centred FP32 (points_to_f32 in indialign_b200/csrc/k_bank.cu), replayed on
the CPU byte for byte: the shared region holds the bulk-copied doubles at
`lead` bytes (0 or 8: the copy starts at the source rounded down to 16
bytes); in round r every thread of the 128-thread CTA first reads point
128r + tid, then (after a barrier) writes it as a float4 (x, y, z, w) at
the start of the region, w = 1 for a valid residue.  No round may overwrite a double that a later read still needs,
and the region must hold the converted set exactly."""
from __future__ import annotations

import numpy as np
import pytest

CTA = 128  # kBankChunk


def _region_bytes(nmax: int) -> int:
    """coord_bytes of k_bank: room for a 15-byte lead and the rounded-up tail."""
    return (nmax * 24 + 47) & ~15


def _replay(points: np.ndarray, lead: int, nmax: int, valid=None) -> np.ndarray:
    n = points.shape[0]
    region = bytearray(_region_bytes(nmax))
    region[lead:lead + 24 * n] = points.astype("<f8").tobytes()
    off = points.mean(0)  # points_mean: FP64 mean of all n points
    for base in range(0, n, CTA):
        idx = range(base, min(base + CTA, n))
        # reads of the round (before the barrier)
        vals = {i: np.frombuffer(bytes(region[lead + 24 * i:lead + 24 * i + 24]), "<f8") for i in idx}
        # writes of the round (after the barrier)
        for i in idx:
            w = 1.0 if valid is None or valid[i] != 0 else 0.0
            region[16 * i:16 * i + 16] = np.append(vals[i] - off, w).astype("<f4").tobytes()
            # every later read lies at or above lead + 24 * (base + CTA)
            assert 16 * i + 16 <= lead + 24 * (base + CTA)
    assert lead + 24 * n <= len(region) and 16 * n <= len(region)
    return np.frombuffer(bytes(region[:16 * n]), "<f4").reshape(n, 4)


@pytest.mark.parametrize("n", [1, 3, 127, 128, 129, 255, 256, 257, 1000, 1500])
@pytest.mark.parametrize("lead", [0, 8])
def test_in_place_conversion_is_exact(n, lead):
    rng = np.random.default_rng(n + lead)
    pts = rng.standard_normal((n, 3)) * 30 + rng.uniform(-50, 50, 3)
    valid = (rng.uniform(size=n) > 0.1).astype(np.uint8) * rng.integers(1, 3, n).astype(np.uint8)
    got = _replay(pts, lead, nmax=n + 7, valid=valid)
    want = (pts - pts.mean(0)).astype(np.float32)
    np.testing.assert_array_equal(got[:, :3], want)
    np.testing.assert_array_equal(got[:, 3], (valid != 0).astype(np.float32))
