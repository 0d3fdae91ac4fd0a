"""The precision study's lowered-precision oracle builds (oracle/precision_study.py):
every textual substitution still applies to the oracle source, every variant
compiles, and on a few small pairs each stays within the per-pair bar of the
reference build (final TM, rescored in FP64, >= reference - 1e-6).  The
bank32 variant is the seed-bank kernel's arithmetic restated on the CPU."""
from __future__ import annotations

import os
import sys

import pytest

from conftest import REF_SO, REF_STAGES_SO, ROOT

sys.path.insert(0, os.path.join(ROOT, "oracle"))
import precision_study as ps  # noqa: E402

from indialign_b200 import workloads as W  # noqa: E402


def test_variant_sources_apply():
    src = open(os.path.join(ROOT, "oracle", "indialign_oracle.c")).read()
    out = ps.variant_sources(src)
    assert sorted(out) == ["bank32", "bank32f", "bank32p", "dist32", "dp32", "kahan32", "plain32", "qcp64", "raw32",
                           "raw32c", "smat32"]
    for name, s in out.items():
        assert s != src, name


@pytest.mark.skipif(not (os.path.exists(REF_SO) and os.path.exists(REF_STAGES_SO)),
                    reason="reference build (oracle/_ref) not present")
def test_variants_stay_within_the_bar(capsys, tmp_path):
    libs = ps.build([], str(tmp_path))
    pairs = W.batch(6, 30, 70, seed=5) + [p for p in W.hard(24, seed=6) if p.pred.shape[0] <= 80][:2]
    ps.compare(pairs, libs, "small")
    out = capsys.readouterr().out
    rows = [l for l in out.splitlines() if "worst" in l]
    assert len(rows) == len(libs)
    for row in rows:
        worst = float(row.split("worst")[1].split()[0])
        assert worst >= -1e-6, row
