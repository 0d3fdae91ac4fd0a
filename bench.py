"""Benchmark of the batched TM-score superposition search (one JSON line).

Workload (default, learned16384): the learned-vs-plain configuration --
16384 synthetic pairs, L ~ U(40,1000), sigma ~ U(0.5,14) A, random rigid
transform, 5 % invalid residues per mask, lnorm = L, default NativeConfig.
A step is one search call over a batch of --step-pairs pairs (4096: four
steps cover the 16384 pairs; warm-up and timed steps take consecutive
batches, cycling through the workload).

  value    pairs/s of the LEARNED search (the rescue passes refine the
           ranker's top-8 candidates per pair, margin 0.02, 2 % audit), inputs
           resident in HBM (indialign_tmscore_search_device), device-timed
           with CUDA events on the call's stream, L2 flushed (256 MB write)
           before every step, max over ranks.
  plain    the PLAIN search (every candidate refined, the reference's
           algorithm) on the first timed batches, one pass over the
           workload's distinct pairs (later timed batches repeat them), same
           timing; its ratio to `value` and the per-pair final TM-score change
           of the learned search against it on every distinct timed pair
           (mean, worst, counts) are reported.
  e2e      the learned search through the C-ABI batch call with host
           buffers: host->device copies of the inputs and the device->host
           read of the results inside the timed region.
  roofline the learned step's two hot kernels (`kernels`), and the larger
           by summed device time as `kernel`: algorithmic flops / device time
           against the GPU's measured FP32 FMA peak (indialign_fp32_peak) --
           seed bank: 55 FP32 flop per residue visit; NW chains: 18 FP32 flop
           per NW cell + 55 FP64 flop per Kabsch / detailed-search residue
           visit, the FP64 flops counted twice (the FP64 rate is half the
           FP32 rate).
  cpu_baseline  the reference's own build (oracle/_ref, OpenMP batch entry)
           on this host's cores: one batch call over a length-stratified
           sample of the timed pairs, two pairs per host thread.

stdout carries one short JSON line (key figures); the full record (ranker
statistics per candidate kind, stage and kernel times, work counters) goes
to stderr and, with --detail-out, to a file.

Multi-GPU (torchrun): pairs are independent, so each rank searches its own
batches of the same shape (weak scaling, no data-path collective); value =
all ranks' pairs / max rank time.  --impl reference: the reference build on
the host cores, rank 0 only: per step one batch call over a stratified
sample of that step's batch, two pairs per host thread and at least 256
timed pairs in all.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from indialign_b200 import abi, workloads as W  # noqa: E402

METRIC = "pairs/sec on 1 B200, learned-seed vs plain GPU search at mean ΔTM ≥ −1e-4"
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libindialign_ref.so")
FLOP_PER_CELL = 18.0
FLOP_PER_VISIT = 55.0
# DRAM bytes (read + write) of the seed-bank kernel per residue visit, from
# an ncu capture (dram__bytes_read.sum + dram__bytes_write.sum) of all nine
# k_bank launches of one 192-pair learned16384 call (`bench.py --step-pairs
# 192 --steps 1 --warmup 0 --no-cpu-baseline --no-e2e --no-plain --no-split`):
# 511.1 MB over that call's 13.08 G residue visits.  The traffic is the item
# records (13 doubles per item) and the staged point sets, which grow in
# proportion to the visits.
BANK_DRAM_BYTES_PER_VISIT = 511.1e6 / 13.084e9
# DRAM bytes (read + write) of the NW chain kernel per NW cell, from the same
# kind of capture of all eleven k_chain launches of one plain batch64 step
# (`bench.py --workload batch64 --mode plain --steps 1 --warmup 0
# --no-cpu-baseline --no-e2e --no-split`): 1.873 GB read + 20.290 GB written
# over that step's 21.999 G NW cells.  Most of it is the chain body's stack
# traffic around its out-of-line calls beside the 2-bit trace; the stack part
# grows with the chain steps rather than the cells, so on longer matrices
# the figure overstates the traffic.
CHAIN_DRAM_BYTES_PER_CELL = 22.163e9 / 21.9986e9
STAGES = ["seeds", "seed_bank", "ss", "gapless", "local_fragment", "threading_dp",
          "dense_local_fragment", "topk", "dp_refine", "offset_dp", "weighted", "total"]


def workload(name: str, step_pairs: int, n_steps: int, rank: int = 0):
    """The pairs of n_steps consecutive batches of `name` for this rank; the
    batches cycle through the workload's pairs (every rank has its own
    workload of the same shape)."""
    if name == "learned16384":
        total = 16384
        n = min(total, step_pairs * n_steps)
        pairs = W.parallel_batch(n, 40, 1000, seed=4 + 1000 * rank)
        desc = ("learned16384: 16384 pairs, L~U(40,1000), sigma~U(0.5,14) A, random rigid transform, "
                f"5% invalid per mask, lnorm=L; a step is one {step_pairs}-pair search call, the steps "
                "cycle through the workload's consecutive batches")
    elif name == "batch4096":
        pairs = W.parallel_batch(min(4096, step_pairs * n_steps), 40, 300, seed=1 + 1000 * rank)
        desc = "batch4096: 4096 pairs, L~U(40,300), sigma~U(0.5,14), 5% invalid per mask"
    elif name == "hard1024":
        pairs = W.hard(1024, seed=2 + 1000 * rank)
        desc = "hard1024: 1024 pairs, L log-uniform 30..1500, half hard (30-60% stems kept)"
    elif name.startswith("batch") and name[5:].isdigit():
        pairs = W.parallel_batch(int(name[5:]), 40, 300, seed=1 + 1000 * rank)
        desc = f"{name}: {len(pairs)} pairs, L~U(40,300), sigma~U(0.5,14), 5% invalid per mask"
    else:
        raise SystemExit(f"unknown workload {name}")
    batches = [pairs[(k * step_pairs) % len(pairs):(k * step_pairs) % len(pairs) + step_pairs]
               for k in range(n_steps)]
    return batches, desc


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        import tempfile
        fd, self.path = tempfile.mkstemp(prefix="indialign_clocks_", suffix=".csv")
        os.close(fd)

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=10)
            self.f.close()

    def summary(self):
        try:
            rows = [l.strip().split(", ") for l in open(self.path) if l.strip()]
            os.remove(self.path)
        except OSError:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(rows)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ref_pairs_per_call(cores: int) -> int:
    """The reference batch entry parallelises over pairs only (one pair per
    OpenMP thread, inner loops serial), so a call needs at least two pairs
    per host thread to keep every core busy until its end."""
    return 2 * cores


def cpu_baseline(pairs, n_sample=0, seed=7):
    """The reference build on this host's cores: one batch call over a
    length-stratified sample of `pairs` with two pairs per host thread."""
    if not os.path.exists(REF_SO):
        return None
    cores = os.cpu_count() or 1
    sample = W.subsample(pairs, n_sample or ref_pairs_per_call(cores), seed=seed)
    os.environ["OMP_NUM_THREADS"] = str(cores)
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    t0 = time.perf_counter()
    _, s, _, _ = abi.run_batch(ref, sample)
    dt = time.perf_counter() - t0
    done, scores = sample, list(s)
    out = {"value": len(done) / dt, "unit": "pairs/s", "cores": cores, "kind": "reference",
           "cpu": cpu_model(),
           "sample": f"one batch call over a {len(sample)}-pair length-stratified sample of the timed "
                     f"pairs (seed {seed}), reference build, OpenMP batch entry, {dt:.1f} s"}
    single = single_thread_rate(done, ref)
    if single:
        out["single_thread"] = single
    return out, done, np.array(scores)


def single_thread_rate(pairs, ref=None, budget_s=8.0):
    """The reference build on ONE host thread: a child process started with
    OMP_NUM_THREADS=1 (the reference's rescue passes are OpenMP-parallel
    inside a single pair) runs the pairs shortest first until `budget_s`;
    with `ref` (the reference library loaded with all cores) the same pairs
    are then timed on all cores, for the parallel speed-up on equal work."""
    import tempfile
    order = sorted(pairs, key=lambda p: p.pred.shape[0])
    fd, path = tempfile.mkstemp(prefix="indialign_single_", suffix=".npz")
    os.close(fd)
    try:
        np.savez(path, **{f"{k}_{i}": np.asarray(getattr(p, k)) for i, p in enumerate(order)
                          for k in ("pred", "native", "valid", "pred_valid", "native_valid")},
                 lnorm=np.array([p.lnorm for p in order]))
        try:
            r = subprocess.run([sys.executable, "-c",
                                f"import bench; bench._single_thread_worker({path!r}, {budget_s})"],
                               cwd=ROOT, env=dict(os.environ, OMP_NUM_THREADS="1"), capture_output=True,
                               text=True, timeout=budget_s + 90)
        except subprocess.TimeoutExpired:
            return {"value": None, "unit": "pairs/s", "cores": 1,
                    "sample": f"the shortest pair did not finish within {budget_s + 90:.0f} s on one thread"}
        if r.returncode != 0 or not r.stdout.strip():
            return None
        out = json.loads(r.stdout.strip().splitlines()[-1])
    finally:
        os.remove(path)
    n = out.pop("pairs")
    lens = [p.pred.shape[0] for p in order[:n]]
    out["sample"] = (f"the {n} shortest pairs (L {min(lens)}-{max(lens)}) of the multi-core sample, "
                     f"one thread, {out.pop('seconds'):.1f} s")
    if ref is not None and n > 0:
        t0 = time.perf_counter()
        abi.run_batch(ref, order[:n])
        out["same_pairs_all_cores"] = n / (time.perf_counter() - t0)
    return out


def _single_thread_worker(path, budget_s):
    z = np.load(path)
    lnorm = z["lnorm"]
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    done, dt = 0, 0.0
    for i in range(len(lnorm)):
        p = W.Pair(*(z[f"{k}_{i}"] for k in ("pred", "native", "valid", "pred_valid", "native_valid")),
                   float(lnorm[i]))
        t0 = time.perf_counter()
        abi.run_batch(ref, [p])
        dt += time.perf_counter() - t0
        done += 1
        if dt >= budget_s:
            break
    print(json.dumps({"value": done / dt if dt > 0 else None, "unit": "pairs/s", "cores": 1,
                      "pairs": done, "seconds": dt}))


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
        return
    batches, desc = workload(args.workload, args.step_pairs, args.warmup + args.steps)
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    # two pairs per host thread per call, and at least 256 timed pairs in all
    per_step = args.ref_pairs or max(ref_pairs_per_call(cores), -(-256 // max(args.steps, 1)))
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    for k in range(args.warmup):
        abi.run_batch(ref, sorted(batches[k], key=lambda p: p.pred.shape[0])[:1])  # shortest pair
    times, n_done = [], 0
    for k in range(args.steps):
        sample = W.subsample(batches[args.warmup + k], per_step, seed=100 + k)
        t0 = time.perf_counter()
        abi.run_batch(ref, sample)
        times.append(time.perf_counter() - t0)
        n_done += len(sample)
    value = n_done / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc,
                       "step": (f"one reference batch call over a {per_step}-pair length-stratified sample "
                                f"of one {args.step_pairs}-pair batch"),
                       "host_threads": cores, "cpu": cpu_model()},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "reference",
                             "cpu": cpu_model(),
                             "sample": f"{per_step} pairs per step x {args.steps} steps = {n_done} pairs"},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def reduce_max(dist, x: float, device: str) -> float:
    """Max of a per-rank time over all ranks (identity without a process
    group); every rank calls it at the same point."""
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(pairs_per_rank: int, world: int, max_ms: float) -> float:
    """pairs/s of the whole job: every rank's pairs over the slowest rank's time."""
    return pairs_per_rank * world / (max_ms / 1e3)


class DeviceBatch:
    """One batch packed back to back in HBM (torch tensors as plumbing)."""

    def __init__(self, torch, pairs):
        self.n = len(pairs)
        lens = [p.pred.shape[0] for p in pairs]
        self.off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)

        def cat(f, dt):
            return torch.from_numpy(np.ascontiguousarray(
                np.concatenate([np.asarray(f(p), dt).reshape(-1) for p in pairs]))).cuda()

        self.pred, self.nat = cat(lambda p: p.pred, np.float64), cat(lambda p: p.native, np.float64)
        self.v, self.pv, self.nv = (cat(lambda p: p.valid, np.uint8), cat(lambda p: p.pred_valid, np.uint8),
                                    cat(lambda p: p.native_valid, np.uint8))
        self.lnorm = np.array([p.lnorm for p in pairs], np.float64)
        self.out = torch.zeros(self.n * 13, dtype=torch.float64, device="cuda")


def plain_steps(batches, steps: int, step_pairs: int) -> int:
    """Timed steps of the plain comparison leg: enough step_pairs-pair calls
    to cover the workload's distinct pairs once (the batches cycle through
    them), at most the learned leg's `steps` and at least one."""
    n_distinct = len({id(p) for b in batches for p in b})
    return max(1, min(steps, -(-n_distinct // max(step_pairs, 1))))


def roofline_record(kern, ctr, step_ms: float, peak: float, peak_source: str) -> dict:
    """The bench line's `roofline` object from one step's mean kernel event
    times (`kern`: k_chain, k_bank, ..., k_rank at index 4; ms) and work
    counters (`ctr`: NW cells, FP64 chain residue visits, seed-bank residue
    visits, ..., warp-cycle split at 8..11).  Both hot kernels are reported,
    algorithmic FP32 flops over their event time (FP64 chain visits counted
    at the FP64 half rate) against `peak` (TFLOP/s), with DRAM traffic per
    step scaled from their captures; the top-level figures are the larger
    kernel's."""
    per_kernel = {
        "k_chain": (FLOP_PER_CELL * ctr[0] + 2.0 * FLOP_PER_VISIT * ctr[1], kern[0],
                    CHAIN_DRAM_BYTES_PER_CELL * ctr[0],
                    "k_chain (NW chains: score matrix + NW + Kabsch + refine)"),
        "k_bank": (FLOP_PER_VISIT * ctr[2], kern[1], BANK_DRAM_BYTES_PER_VISIT * ctr[2],
                   "k_bank (seed x cutoff refine items)"),
    }
    top = "k_chain" if kern[0] >= kern[1] else "k_bank"
    flops, kms, traffic, kname = per_kernel[top]
    achieved = flops / (kms / 1e3) / 1e12 if kms > 0 else None
    both = {}
    for nm, (fl, ms, tr, _) in per_kernel.items():
        ach = fl / (ms / 1e3) / 1e12 if ms > 0 else None
        both[nm] = {"ms_per_step": round(float(ms), 1), "achieved": ach,
                    "frac": ach / peak if ach else None, "traffic": tr}
    cyc = np.asarray(ctr[8:12], dtype=np.float64)
    return {"kernel": kname, "bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None, "traffic": traffic,
            "traffic_unit": "bytes per step (DRAM read + write of the kernel's launches)",
            "peak_source": peak_source,
            "kernel_ms_per_step": float(kms), "kernel_share": float(kms / step_ms),
            "kernels": both,
            "kernel_ms": {"k_chain": float(kern[0]), "k_bank": float(kern[1]), "k_rank": float(kern[4])},
            "nw_cells_per_step": int(ctr[0]), "chain_visits_per_step": int(ctr[1]),
            "bank_visits_per_step": int(ctr[2]),
            "warp_cycle_split": dict(zip(["nw_fill", "traceback", "detailed", "kabsch"],
                                         [float(x) for x in cyc / max(1.0, cyc.sum())]))}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="learned16384")
    ap.add_argument("--mode", default="learned", choices=["learned", "plain"],
                    help="search timed for `value`; with learned, the plain search is timed beside it")
    ap.add_argument("--step-pairs", type=int, default=4096,
                    help="pairs per search call (default: 4 timed steps cover the 16384-pair workload once)")
    ap.add_argument("--top-k", type=int, default=8)
    ap.add_argument("--margin", type=float, default=0.02)
    ap.add_argument("--audit", type=float, default=0.02)
    ap.add_argument("--rank-mask", type=int, default=0, help="INDIALIGN_RANK_* bits (0: library default)")
    ap.add_argument("--weights", default=None, help="ranker blob (.npy; default the shipped weights)")
    ap.add_argument("--ref-pairs", type=int, default=0,
                    help="pairs per reference-arm step (0: two per host thread, >= 256 timed in all)")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="pairs of the cpu_baseline call (0: two per host thread)")
    ap.add_argument("--detail-out", default=None, help="also write the full record (JSON) here")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-split", action="store_true",
                    help="run every call as one batch (the kernel-shape table's split flag off), e.g. so that "
                         "a profiler's launch numbering follows one search's stage order")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    batches, desc = workload(args.workload, args.step_pairs, args.warmup + args.steps, rank)

    import torch
    import indialign_b200 as ia
    from indialign_b200 import ranker

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    lib = ia.load()
    if args.no_split:
        ia.set_tuning(dict(ia.get_tuning(), split=0))
    cfg = ia.default_config()
    blob = (np.ascontiguousarray(np.load(args.weights), np.float32) if args.weights
            else ranker.default_weights())
    dev = [DeviceBatch(torch, b) for b in batches]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def make_opts(learned: bool):
        o = ia.BatchOptions()
        o.device = local
        o.stream = ctypes.c_void_p(stream.cuda_stream)
        o.kern = np.zeros(6)
        o.ctr = np.zeros(12, np.int64)
        o.stg = np.zeros(12)
        o.rst = np.zeros(ia.RANK_STATS, np.int64)
        o.kernel_ms = o.kern.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        o.counters = o.ctr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
        o.stage_ms = o.stg.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        if learned:
            ia.learned_options(o, blob, args.top_k, args.margin, args.audit, 1234 + rank, o.rst,
                               args.rank_mask)
        return o

    def device_step(db, o):
        rc = lib.indialign_tmscore_search_device(
            db.n, db.off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), db.pred.data_ptr(), db.nat.data_ptr(),
            db.v.data_ptr(), db.pv.data_ptr(), db.nv.data_ptr(),
            db.lnorm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(cfg), ctypes.byref(o),
            db.out.data_ptr())
        if rc != 0:
            raise SystemExit(f"search failed rc={rc}: {ia.last_error()}")

    def barrier():
        if dist:
            dist.barrier()

    def timed(fn):
        flush.zero_()
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1)

    def run_mode(learned: bool, clocks=None, steps=None, warmup=None):
        o = make_opts(learned)
        for k in range(args.warmup if warmup is None else warmup):
            timed(lambda: device_step(dev[k], o))
        rec = dict(ms=[], kern=[], ctr=[], stg=[], rst=[], scores=[])
        ctx = clocks if clocks is not None else _Null()
        with ctx:
            for k in range(args.steps if steps is None else steps):
                db = dev[args.warmup + k]
                rec["ms"].append(timed(lambda: device_step(db, o)))
                rec["kern"].append(o.kern.copy())
                rec["ctr"].append(o.ctr.copy())
                rec["stg"].append(o.stg.copy())
                rec["rst"].append(o.rst.copy())
                rec["scores"].append(db.out.view(db.n, 13)[:, 0].cpu().numpy())
        return rec

    def max_over_ranks(x):
        return reduce_max(dist, x, "cuda")

    learned_mode = args.mode == "learned"
    clk = Clocks(local)
    lrn = run_mode(learned_mode, clk)
    clocks = clk.summary()
    n_timed = sum(dev[args.warmup + k].n for k in range(args.steps))
    l_ms = max_over_ranks(float(np.sum(lrn["ms"])))
    value = whole_job_rate(n_timed, world, l_ms)
    l_scores = np.concatenate(lrn["scores"])

    plain = None
    if learned_mode and not args.no_plain:
        # the plain search on the first timed batches, one pass over the
        # workload's distinct pairs (later timed batches repeat them, and a
        # pair's results do not change between calls), after min(W, 3)
        # warm-up steps: its throughput and the learned search's TM change
        # on every distinct timed pair
        p_steps = plain_steps(batches, args.steps, args.step_pairs)
        pl = run_mode(False, steps=p_steps, warmup=min(args.warmup, 3))
        p_n = sum(dev[args.warmup + k].n for k in range(p_steps))
        p_ms = max_over_ranks(float(np.sum(pl["ms"])))
        p_scores = np.concatenate(pl["scores"])
        d = l_scores[:p_n] - p_scores
        l_rate = n_timed * world / (l_ms / 1e3)
        plain = {"value": p_n * world / (p_ms / 1e3), "unit": "pairs/s", "steps": p_steps,
                 "ms_per_step": p_ms / p_steps, "learned_over_plain": l_rate / (p_n * world / (p_ms / 1e3)),
                 "delta_tm": {"mean": float(d.mean()), "worst": float(d.min()), "best": float(d.max()),
                              "pairs_below_-1e-4": int(np.sum(d < -1e-4)),
                              "pairs_below_-1e-3": int(np.sum(d < -1e-3)), "pairs": int(d.size)},
                 "stage_ms": dict(zip(STAGES, [round(float(x), 2) for x in np.mean(pl["stg"], 0)])),
                 "kernel_ms": {"k_chain": float(np.mean([k[0] for k in pl["kern"]])),
                               "k_bank": float(np.mean([k[1] for k in pl["kern"]]))}}
    else:
        p_scores = None

    # end to end: the learned search through the C-ABI batch entry with host buffers
    e2e = None
    if not args.no_e2e:
        eo = make_opts(learned_mode)
        eo.kernel_ms = eo.counters = eo.stage_ms = None
        packs = [abi.PackedInputs(b) for b in batches[args.warmup:args.warmup + args.steps]]
        res = [(abi.NativePairResult * p.n)() for p in packs]
        timed(lambda: lib.indialign_tmscore_search_batch_ex(packs[0].n, packs[0].arr, ctypes.byref(cfg),
                                                            ctypes.byref(eo), res[0]))
        et = []
        for k, pk in enumerate(packs):
            rc = []
            et.append(timed(lambda: rc.append(lib.indialign_tmscore_search_batch_ex(
                pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(eo), res[k]))))
            assert rc[0] == 0, ia.last_error()
        es = np.concatenate([abi.results_to_numpy(r, p.n)[0] for r, p in zip(res, packs)])
        assert np.array_equal(es, l_scores), "host and device entry points disagree"
        e_ms = max_over_ranks(float(np.sum(et)))
        pairs_t = [p for b in batches[args.warmup:] for p in b]
        h2d = int(sum(p.pred.shape[0] * (48 + 3) + 8 for p in pairs_t)) // args.steps
        e2e = {"value": n_timed * world / (e_ms / 1e3), "unit": "pairs/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": 104 * n_timed // args.steps}

    if rank == 0:
        kern = np.mean(lrn["kern"], 0)
        ctr = np.mean(lrn["ctr"], 0)
        step_ms = l_ms / args.steps
        peak = ia.fp32_peak_tflops(local)
        roofline = roofline_record(kern, ctr, step_ms, peak,
                                   "measured FP32 FMA rate (indialign_fp32_peak) in this run")
        # the library counts its stage launches (counter 7); the device entry
        # adds the input repack and the result export, the learned search the
        # MLP weight pack
        per_call = 2 + (1 if learned_mode else 0)
        launches = int(sum(int(c[7]) + per_call for c in lrn["ctr"]))
        rst = np.sum(lrn["rst"], 0).reshape(ia.CAND_KINDS, -1)
        rank_info = {}
        for k, nm in enumerate(ia.CAND_NAMES):
            g = max(int(rst[k, 0]), 1)
            rank_info[nm] = {"pairs": int(rst[k, 0]), "fallback_rate": rst[k, 1] / g, "audit_rate": rst[k, 2] / g,
                             "pruned_rate": rst[k, 3] / g, "refined_fraction": rst[k, 5] / max(int(rst[k, 4]), 1),
                             "audits": int(rst[k, 2]), "audit_misses": int(rst[k, 6]),
                             "audit_misses_1e-4": int(rst[k, 8]), "audit_misses_1e-3": int(rst[k, 9])}
        cpu = None
        if not args.no_cpu_baseline:
            timed_pairs = [p for b in batches[args.warmup:] for p in b]
            r = cpu_baseline(timed_pairs, args.cpu_sample)
            if r:
                cpu, done, ref_s = r
                if p_scores is not None:
                    pos = {id(p): k for k, p in enumerate(timed_pairs)}
                    idx = [pos[id(p)] for p in done]
                    d = p_scores[idx] - ref_s
                    cpu["plain_parity_on_sample"] = {"min_dTM": float(d.min()),
                                                     "max_abs_dTM": float(np.abs(d).max()),
                                                     "pairs_below_ref_minus_1e-6": int(np.sum(d < -1e-6))}
        line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f64+f32 (seed-bank residue visits f32)", "data": "synthetic",
                "config": {"workload": desc, "step_pairs": args.step_pairs, "pairs_timed_per_gpu": n_timed,
                           "mode": (f"learned (top_k {args.top_k}, margin {args.margin}, audit {args.audit}, "
                                    f"rank_mask {args.rank_mask or 'default'})"
                                    if learned_mode else "plain"),
                           "ranker": "indialign_b200/ranker_weights.npy",
                           "l2": "flushed by a 256 MB write before every step",
                           "parallelism": f"independent pairs per GPU x{world}"},
                "plain": plain, "rank": rank_info, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "gpu_launches_per_step": launches / args.steps, "clocks": clocks,
                "stage_ms": dict(zip(STAGES, [round(float(x), 2) for x in np.mean(lrn["stg"], 0)])),
                "mean_tm": float(l_scores.mean())}
        # the full record goes to stderr (and --detail-out); stdout gets one
        # short line whose every key survives a few-KB tail of the output
        print(json.dumps(line), file=sys.stderr)
        if args.detail_out:
            with open(args.detail_out, "w") as f:
                json.dump(line, f, indent=1)
        print(json.dumps(compact_line(line)))
    if dist:
        dist.destroy_process_group()


def compact_line(line: dict) -> dict:
    """The bench line without the per-kind ranker statistics, stage and
    kernel breakdowns (those stay in the full record): key figures first."""
    keep = ["metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
            "scaling", "vs_baseline", "dtype", "data"]
    out = {k: line[k] for k in keep}
    pl = line.get("plain")
    if pl:
        out["plain"] = {k: pl[k] for k in ("value", "unit", "steps", "ms_per_step", "learned_over_plain", "delta_tm")
                        if k in pl}
    if line.get("rank"):
        r = line["rank"]
        lists = sum(v["pairs"] for v in r.values())
        out["rank"] = {"lists": lists,
                       "fallback_rate": sum(v["fallback_rate"] * v["pairs"] for v in r.values()) / max(lists, 1),
                       "audits": sum(v.get("audits", 0) for v in r.values()),
                       "audit_misses": sum(v["audit_misses"] for v in r.values()),
                       "audit_misses_1e-4": sum(v.get("audit_misses_1e-4", 0) for v in r.values()),
                       "miss_rate_1e-4": {k: round(v.get("audit_misses_1e-4", 0) / v["audits"], 3)
                                          for k, v in r.items() if v.get("audits")}}
    rf = line.get("roofline")
    if rf:
        out["roofline"] = {k: rf[k] for k in ("kernel", "bound", "achieved", "peak", "unit", "frac", "traffic",
                                              "peak_source", "kernel_share", "kernels") if k in rf}
    cpu = line.get("cpu_baseline")
    if cpu:
        out["cpu_baseline"] = {k: v for k, v in cpu.items() if k != "single_thread"}
        st = cpu.get("single_thread")
        if st:
            out["cpu_baseline"]["single_thread"] = {"value": st.get("value"), "cores": 1}
    for k in ("e2e", "gpu_launches", "mean_tm", "config"):
        out[k] = line.get(k)
    c = line.get("clocks")
    out["clocks"] = {k: c[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")} if c else None
    return out


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
