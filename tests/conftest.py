"""Shared fixtures: the product library, the oracle (C restatement) and, when
it was built here, the reference's own build; golden fixture loaders."""
from __future__ import annotations

import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from indialign_b200 import abi, workloads  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden")
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libindialign_ref.so")
REF_STAGES_SO = os.path.join(ROOT, "oracle", "_ref", "libindialign_ref_stages.so")
LIB_SO = os.path.join(ROOT, "indialign_b200", "libindialign.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built(path, target_dir, target):
    if not os.path.exists(path):
        subprocess.run(["make", "-s", "-C", target_dir, target], check=True)


@pytest.fixture(scope="session")
def oracle():
    _ensure_built(ORACLE_SO, os.path.join(ROOT, "oracle"), "oracle")
    return abi.bind_reference_abi(ctypes.CDLL(ORACLE_SO), prefix="ora_")


@pytest.fixture(scope="session")
def ref():
    if not os.path.exists(REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    return abi.bind_reference_abi(ctypes.CDLL(REF_SO))


@pytest.fixture(scope="session")
def ref_stages():
    if not os.path.exists(REF_STAGES_SO):
        pytest.skip("reference stage wrappers (oracle/_ref) not present")
    return ctypes.CDLL(REF_STAGES_SO)


class GoldenPairs:
    """Pairs and reference results of one golden fixture file."""

    def __init__(self, name):
        z = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
        self.name = name
        off = z["off"]
        self.pairs = []
        for k in range(len(off) - 1):
            a, b = int(off[k]), int(off[k + 1])
            self.pairs.append(workloads.Pair(
                z["pred"][3 * a:3 * b].reshape(-1, 3), z["nat"][3 * a:3 * b].reshape(-1, 3),
                z["v"][a:b], z["pv"][a:b], z["nv"][a:b], float(z["lnorm"][k]),
                float(z["sigma"][k])))
        self.score, self.R, self.t, self.trace = z["score"], z["R"], z["t"], z["trace"]
        self.hard = z["hard"] if "hard" in z else np.zeros(len(self.pairs), bool)

    def shortest(self, k):
        """Indices of the k shortest pairs (for checks that must stay fast on
        the CPU)."""
        return sorted(range(len(self.pairs)), key=lambda i: self.pairs[i].pred.shape[0])[:k]


GOLDEN_SETS = ["single", "batch", "hard", "edge"]


@pytest.fixture(scope="session", params=GOLDEN_SETS)
def golden(request):
    return GoldenPairs(request.param)


def rot_err_deg(R1, R2):
    """Angle (degrees) of R1^T R2 for flattened 3x3 rotations."""
    out = []
    for a, b in zip(R1, R2):
        M = a.reshape(3, 3).T @ b.reshape(3, 3)
        c = np.clip((np.trace(M) - 1) / 2, -1.0, 1.0)
        out.append(np.degrees(np.arccos(c)))
    return np.array(out)
