"""The device eigen-solve (characteristic polynomial of Horn's key matrix,
the reference's Jacobi sequence for near-degenerate top eigenvalues) against
the oracle's restatement of the reference's cov_to_rotation
(indialign_c/core.h:29-90), through the C ABI self-test entry."""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import ORACLE_SO

import indialign_b200 as ia


def _rotation(rng):
    a = rng.standard_normal((3, 3))
    q, r = np.linalg.qr(a)
    q *= np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] *= -1
    return q


def _horn(h):
    """Horn's key matrix of a covariance (indialign_c/core.h:64-75)."""
    return np.array([
        [h[0, 0] + h[1, 1] + h[2, 2], h[1, 2] - h[2, 1], h[2, 0] - h[0, 2], h[0, 1] - h[1, 0]],
        [h[1, 2] - h[2, 1], h[0, 0] - h[1, 1] - h[2, 2], h[0, 1] + h[1, 0], h[2, 0] + h[0, 2]],
        [h[2, 0] - h[0, 2], h[0, 1] + h[1, 0], -h[0, 0] + h[1, 1] - h[2, 2], h[1, 2] + h[2, 1]],
        [h[0, 1] - h[1, 0], h[2, 0] + h[0, 2], h[1, 2] + h[2, 1], -h[0, 0] - h[1, 1] + h[2, 2]]])


def _covariances(n, seed=11):
    """Centred covariances of point sets: general, near-planar, near-linear
    and very noisy, plus exact special cases."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        m = int(rng.integers(3, 300))
        p = rng.standard_normal((m, 3)) * rng.uniform(1, 30)
        if k % 4 == 1:
            p[:, 2] *= 1e-6
        if k % 4 == 2:
            p[:, 1:] *= 1e-6
        q = p @ _rotation(rng) + rng.standard_normal((m, 3)) * rng.uniform(0, 10 if k % 4 != 3 else 100)
        out.append((p - p.mean(0)).T @ (q - q.mean(0)))
    out += [np.eye(3), np.diag([3.0, 2.0, 1.0]), np.diag([1.0, 1.0, -1.0]), np.zeros((3, 3)),
            np.outer([1.0, 2.0, 3.0], [0.5, -1.0, 2.0])]
    return np.ascontiguousarray(np.array(out).reshape(-1, 9))


@pytest.mark.gpu
def test_device_rotation_matches_reference_cov_to_rotation():
    H = _covariances(4000)
    n = H.shape[0]
    R = np.zeros_like(H)
    lib = ia.load()
    f = lib.indialign_selftest_rotation
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    assert f(n, H.ctypes.data, R.ctypes.data) == 0, ia.last_error()
    ora = ctypes.CDLL(ORACLE_SO)
    ora.ora_cov_to_rotation.restype = None
    Ro = np.zeros_like(H)
    for i in range(n):
        ora.ora_cov_to_rotation(ctypes.c_void_p(H[i].ctypes.data), ctypes.c_void_p(Ro[i].ctypes.data))
    # where the top eigenvalue of Horn's matrix is separated the rotation is
    # unique: the device's must be the reference's; inside a (near-)
    # degenerate top pair any vector of the pair is optimal, so there both
    # must reach the same objective sum_kd R_kd H_kd (= the top eigenvalue)
    lam = np.array([np.linalg.eigvalsh(_horn(h.reshape(3, 3))) for h in H])
    scale = np.sqrt((lam ** 2).sum(1))
    separated = lam[:, 3] - lam[:, 2] >= 1e-3 * np.maximum(scale, 1e-300)
    assert separated.sum() > 0.6 * n
    err = np.abs(R - Ro).max(1)
    assert err[separated].max() < 1e-9, (err[separated].max(), int(np.argmax(np.where(separated, err, 0))))
    obj, obj_o = (R * H).sum(1), (Ro * H).sum(1)
    assert np.all(obj >= obj_o - 1e-9 * np.maximum(scale, 1.0)), np.min(obj - obj_o)
    M = R.reshape(n, 3, 3)
    assert np.abs(np.einsum("nij,nkj->nik", M, M) - np.eye(3)).max() < 1e-12
    assert np.abs(np.linalg.det(M) - 1.0).max() < 1e-12
