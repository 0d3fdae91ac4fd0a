"""bench.py pieces that need no GPU: the reference arm (the reference build on
the host cores) and its one-line JSON contract, rank gating under torchrun,
the workload batching, and the clock-record parsing."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

from conftest import REF_SO, ROOT

sys.path.insert(0, ROOT)
import bench  # noqa: E402

ARGS = ["--impl", "reference", "--workload", "batch12", "--step-pairs", "4", "--steps", "2", "--warmup", "1",
        "--ref-pairs", "2"]


def _run(env_extra):
    env = dict(os.environ, OMP_NUM_THREADS="2", **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *ARGS], env=env, cwd=ROOT,
                          capture_output=True, text=True, timeout=600)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
def test_reference_arm_json_line():
    r = _run({})
    assert r.returncode == 0, r.stderr
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["metric"] == bench.METRIC
    assert d["unit"] == "pairs/s" and d["higher_is_better"] is True and d["value"] > 0
    assert d["steps"] == 2 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert d["config"]["workload"].startswith("batch12")


def test_reference_arm_other_ranks_do_nothing():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_workload_batches():
    batches, desc = bench.workload("batch10", 4, 3)
    assert [len(b) for b in batches] == [4, 4, 2]  # consecutive slices of the 10 pairs
    assert desc.startswith("batch10")
    b1, _ = bench.workload("batch10", 4, 3, rank=1)
    assert b1[0][0].pred.shape != batches[0][0].pred.shape or \
        (b1[0][0].pred != batches[0][0].pred).any()  # ranks draw their own pairs
    with pytest.raises(SystemExit):
        bench.workload("nonsense", 4, 1)


def test_clock_summary_parsing():
    c = bench.Clocks(0)
    rows = ["0, 1965, 1965, 640.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 700.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
            "0, 1800, 1965, 710.0, 0x0000000000000008, Active, Not Active, Not Active, Active"]
    with open(c.path, "w") as f:
        f.write("\n".join(rows) + "\n")
    s = c.summary()
    assert s["sm_mhz"] == 1950 and s["sm_max_mhz"] == 1965 and s["samples"] == 3
    assert s["reasons"] == ["hw_slowdown", "sw_power_cap"]
    assert not os.path.exists(c.path)


def test_whole_job_rate_and_reduce_without_group():
    assert bench.whole_job_rate(100, 4, 2000.0) == pytest.approx(200.0)
    assert bench.reduce_max(None, 3.5, "cpu") == 3.5


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference build (oracle/_ref) not present")
def test_single_thread_reference_rate():
    from indialign_b200 import workloads
    pairs = workloads.batch(3, 30, 50, seed=5)
    import ctypes
    from indialign_b200 import abi
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    r = bench.single_thread_rate(pairs, ref, budget_s=0.5)
    assert r["cores"] == 1 and r["unit"] == "pairs/s" and r["value"] > 0
    assert r["same_pairs_all_cores"] > 0 and "shortest" in r["sample"]
