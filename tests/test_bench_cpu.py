"""bench.py pieces that need no GPU: the reference arm (the reference build on
the host cores) and its one-line JSON contract, rank gating under torchrun,
the workload batching, the clock-record parsing and the roofline record."""
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


def test_plain_leg_covers_the_distinct_pairs_once():
    # 3 warm-up + 4 timed batches of 4 cycling through 12 pairs: 3 plain steps
    batches, _ = bench.workload("batch12", 4, 7)
    assert bench.plain_steps(batches, 4, 4) == 3
    timed = [id(p) for b in batches[3:3 + 3] for p in b]
    assert len(set(timed)) == 12 and len(timed) == 12  # the first 3 timed batches hold every pair once
    assert bench.plain_steps(batches, 2, 4) == 2       # never more than the learned leg's steps
    assert bench.plain_steps(batches[:1], 4, 64) == 1


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


def test_compact_line_keeps_the_key_fields_in_a_short_line():
    """stdout's line keeps the learned-vs-plain ratio and the per-pair TM
    change, the roofline, the CPU baseline, e2e and clocks, and stays well
    under a few-KB output tail even with the full record's breakdowns."""
    kinds = {nm: {"pairs": 1000 + k, "fallback_rate": 0.1, "audit_rate": 0.02, "pruned_rate": 0.8,
                  "refined_fraction": 0.2, "audit_misses": 7} for k, nm in enumerate("abcde")}
    full = {"metric": bench.METRIC, "value": 1786.0, "unit": "pairs/s", "n_gpus": 1, "steps": 20, "warmup": 5,
            "ms_per_step": 1146.6, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32", "data": "synthetic",
            "config": {"workload": "learned16384: " + "x" * 200, "step_pairs": 2048},
            "plain": {"value": 405.0, "unit": "pairs/s", "ms_per_step": 5059.0, "learned_over_plain": 4.41,
                      "delta_tm": {"mean": 4e-8, "worst": -5e-7, "best": 1e-3, "pairs_below_-1e-4": 0,
                                   "pairs_below_-1e-3": 0, "pairs": 40960},
                      "stage_ms": {s: 1.0 for s in bench.STAGES}, "kernel_ms": {"k_chain": 1.0}},
            "rank": kinds,
            "roofline": {"kernel": "k_bank", "bound": "fp32", "achieved": 12.0, "peak": 67.7, "unit": "TFLOP/s",
                         "frac": 0.18, "traffic": 1.0e9, "peak_source": "measured", "kernel_share": 0.55,
                         "warp_cycle_split": {"nw_fill": 0.8}, "kernel_ms": {"k_bank": 1.0}},
            "cpu_baseline": {"value": 0.9, "unit": "pairs/s", "cores": 16, "kind": "reference", "cpu": "Xeon",
                             "sample": "s" * 150, "single_thread": {"value": 0.45, "sample": "t" * 100},
                             "plain_parity_on_sample": {"min_dTM": -1e-8}},
            "e2e": {"value": 1733.0, "unit": "pairs/s", "h2d_bytes_per_step": 54540422,
                    "d2h_bytes_per_step": 212992},
            "gpu_launches": 3140, "gpu_launches_per_step": 157.0,
            "clocks": {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 108},
            "stage_ms": {s: 1.0 for s in bench.STAGES}, "mean_tm": 0.48}
    c = bench.compact_line(full)
    text = json.dumps(c)
    assert len(text) < 2000
    assert c["plain"]["delta_tm"]["worst"] == -5e-7 and c["plain"]["learned_over_plain"] == 4.41
    assert c["roofline"]["frac"] == 0.18 and c["roofline"]["traffic"] == 1.0e9
    assert c["cpu_baseline"]["cpu"] == "Xeon" and c["e2e"]["value"] == 1733.0
    assert c["rank"]["lists"] == sum(v["pairs"] for v in kinds.values())
    assert list(c)[:3] == ["metric", "value", "unit"]


def test_roofline_record_from_counters():
    """Both hot kernels' figures come from the step's work counters and event
    times: algorithmic flops per unit x units / time against the peak, and
    DRAM traffic scaled from each kernel's capture by the same units; the
    top-level figures are the larger kernel's."""
    kern = [600.0, 750.0, 0.0, 0.0, 120.0]        # ms per step: k_chain, k_bank, ..., k_rank
    ctr = [2.0e10, 1.0e9, 2.5e11, 0, 0, 0, 0, 150, 3.0, 1.0, 0.0, 0.0]
    r = bench.roofline_record(kern, ctr, 1400.0, 67.5, "measured")
    bank = 55.0 * 2.5e11 / 0.75 / 1e12
    chain = (18.0 * 2.0e10 + 2 * 55.0 * 1.0e9) / 0.6 / 1e12
    assert r["kernel"].startswith("k_bank") and r["achieved"] == pytest.approx(bank)
    assert r["frac"] == pytest.approx(bank / 67.5) and r["kernel_share"] == pytest.approx(750 / 1400)
    assert r["traffic"] == pytest.approx(bench.BANK_DRAM_BYTES_PER_VISIT * 2.5e11)
    k = r["kernels"]
    assert k["k_chain"]["achieved"] == pytest.approx(chain)
    assert k["k_chain"]["traffic"] == pytest.approx(bench.CHAIN_DRAM_BYTES_PER_CELL * 2.0e10)
    assert 1.0 < bench.CHAIN_DRAM_BYTES_PER_CELL < 1.02 and 0.03 < bench.BANK_DRAM_BYTES_PER_VISIT < 0.05
    assert r["warp_cycle_split"]["nw_fill"] == pytest.approx(0.75)
    # the plain step: the chain kernel is the larger one
    r2 = bench.roofline_record([6000.0, 10.0, 0, 0, 0], ctr, 7000.0, 67.5, "measured")
    assert r2["kernel"].startswith("k_chain") and r2["traffic"] == k["k_chain"]["traffic"]


def test_reference_arm_fills_the_host():
    """Two pairs per host thread per reference call."""
    assert bench.ref_pairs_per_call(16) == 32
