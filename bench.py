"""Benchmark of the batched TM-score superposition search (one JSON line).

Workload (default): batch4096 -- 4096 synthetic pairs, L ~ U(40,300),
sigma ~ U(0.5,14) A, random rigid transform, 5 % invalid per mask, lnorm = L,
default NativeConfig.  A step is one search over the whole batch.

  value  pairs/s with inputs resident in HBM (indialign_tmscore_search_device),
         device-timed with CUDA events on the call's stream, L2 flushed
         (256 MB write) between steps, max over ranks.
  e2e    the same through the C-ABI batch call with host buffers: the
         host->device copy of the inputs and the device->host read of the
         results are inside the timed region.
  roofline  for the NW-chain kernel (the dominant kernel): algorithmic FP64
         flops (18 per NW cell: 13 score-matrix + 5 DP; 55 per Kabsch/refine
         residue visit) / its summed device time, against the measured FP64
         FMA peak of the GPU (indialign_fp64_peak).
  cpu_baseline  the reference's own build (oracle/_ref, OpenMP batch entry)
         on this host's cores, on a stratified subsample of the workload.

Multi-GPU (torchrun): pairs are independent, so each rank searches its own
batch of the same shape (weak scaling, no data-path collective); value = all
ranks' pairs / max rank time.  --impl reference: the reference build on the
host cores, rank 0 only.
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


def workload(name: str, seed_shift: int = 0):
    if name == "batch4096":
        return W.batch(4096, 40, 300, seed=1 + seed_shift), \
            "batch4096: 4096 pairs, L~U(40,300), sigma~U(0.5,14), 5% invalid per mask"
    if name == "hard1024":
        return W.hard(1024, seed=2 + seed_shift), \
            "hard1024: 1024 pairs, L log-uniform 30..1500, half hard (30-60% stems kept)"
    if name == "single":
        return W.single(0), "single: L=64, sigma=2.0, all valid"
    if name.startswith("batch"):
        n = int(name[5:])
        return W.batch(n, 40, 300, seed=1 + seed_shift), f"batch{n}: L~U(40,300), sigma~U(0.5,14)"
    raise SystemExit(f"unknown workload {name}")


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out" if os.path.isdir(os.path.join(ROOT, "gpurun_out")) else ".",
                                 f".clocks_{os.getpid()}.csv")

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


def cpu_baseline(pairs, n_sample=64, seed=7):
    """The reference build on this host's cores over a stratified subsample."""
    if not os.path.exists(REF_SO):
        return None
    sample = W.subsample(pairs, n_sample, seed=seed)
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    t0 = time.perf_counter()
    rc, s, _, _ = abi.run_batch(ref, sample)
    dt = time.perf_counter() - t0
    return {"value": len(sample) / dt, "unit": "pairs/s", "cores": cores, "kind": "reference",
            "sample": f"{len(sample)}-pair length-stratified subsample of the workload (seed {seed}), "
                      f"reference build, OpenMP batch entry, {dt:.1f} s"}, sample, s


def run_reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    pairs, desc = workload(args.workload)
    if not os.path.exists(REF_SO):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref not present"}))
        return
    cores = os.cpu_count() or 1
    os.environ["OMP_NUM_THREADS"] = str(cores)
    ref = abi.bind_reference_abi(ctypes.CDLL(REF_SO))
    warm = W.subsample(pairs, 4, seed=3)
    for _ in range(args.warmup):
        abi.run_batch(ref, warm)
    times, n_done = [], 0
    for k in range(args.steps):
        sample = W.subsample(pairs, args.ref_pairs, seed=100 + k)
        t0 = time.perf_counter()
        abi.run_batch(ref, sample)
        times.append(time.perf_counter() - t0)
        n_done += len(sample)
    value = n_done / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "pairs/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": desc, "step": f"{args.ref_pairs}-pair stratified subsample per step",
                       "host_threads": cores},
            "cpu_baseline": {"value": value, "unit": "pairs/s", "cores": cores, "kind": "reference",
                             "sample": f"{args.ref_pairs} pairs per step x {args.steps} steps"},
            "e2e": {"value": value, "unit": "pairs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch4096")
    ap.add_argument("--ref-pairs", type=int, default=48)
    ap.add_argument("--cpu-sample", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    import torch
    import indialign_b200 as ia

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    pairs, desc = workload(args.workload, seed_shift=1000 * rank)
    n = len(pairs)
    lib = ia.load()
    cfg = ia.default_config()
    # inputs resident in HBM
    lens = [p.pred.shape[0] for p in pairs]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int32)
    cat = lambda f, dt: torch.from_numpy(np.ascontiguousarray(
        np.concatenate([np.asarray(f(p), dt).reshape(-1) for p in pairs]))).cuda()
    d_pred, d_nat = cat(lambda p: p.pred, np.float64), cat(lambda p: p.native, np.float64)
    d_v, d_pv, d_nv = (cat(lambda p: p.valid, np.uint8), cat(lambda p: p.pred_valid, np.uint8),
                       cat(lambda p: p.native_valid, np.uint8))
    lnorm = np.array([p.lnorm for p in pairs], np.float64)
    d_out = torch.zeros(n * 13, dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    kern = np.zeros(6)
    ctr = np.zeros(12, np.int64)
    stage_ms = np.zeros(12)
    opts = ia.BatchOptions()
    opts.device = local
    opts.stream = ctypes.c_void_p(stream.cuda_stream)
    opts.kernel_ms = kern.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    opts.counters = ctr.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    opts.stage_ms = stage_ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))

    def step():
        rc = lib.indialign_tmscore_search_device(
            n, off.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), d_pred.data_ptr(), d_nat.data_ptr(),
            d_v.data_ptr(), d_pv.data_ptr(), d_nv.data_ptr(),
            lnorm.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(cfg),
            ctypes.byref(opts), d_out.data_ptr())
        if rc != 0:
            raise SystemExit(f"search failed rc={rc}: {ia.last_error()}")

    def barrier():
        if dist:
            dist.barrier()

    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize()
    times, kms, cells, visits, launches, cyc, stg = [], [], [], [], [], [], []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            times.append(e0.elapsed_time(e1))
            kms.append(kern[0])
            cells.append(ctr[0])
            visits.append(ctr[1])
            launches.append(int(ctr[7]) + 2)  # + repack and export
            cyc.append(ctr[8:12].copy())
            stg.append(stage_ms.copy())
    clocks = clk.summary()
    ms = float(np.mean(times))
    t_max = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    ms_max = float(t_max.item())
    value = n * world / (ms_max / 1e3)
    scores = d_out.view(n, 13)[:, 0].cpu().numpy()

    # end to end through the C-ABI batch entry (host buffers)
    e2e = None
    if not args.no_e2e:
        pk = abi.PackedInputs(pairs)
        res = (abi.NativePairResult * n)()
        eopts = ia.BatchOptions()
        eopts.device = local
        eopts.stream = ctypes.c_void_p(stream.cuda_stream)
        etimes = []
        for k in range(1 + min(args.steps, 2)):
            flush.zero_()
            torch.cuda.synchronize()
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.indialign_tmscore_search_batch_ex(n, pk.arr, ctypes.byref(cfg), ctypes.byref(eopts), res)
            e1.record(stream)
            torch.cuda.synchronize()
            barrier()
            assert rc == 0, ia.last_error()
            if k > 0:
                etimes.append(e0.elapsed_time(e1))
        em = torch.tensor([float(np.mean(etimes))], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(em, op=dist.ReduceOp.MAX)
        es, _, _ = abi.results_to_numpy(res, n)
        assert np.array_equal(es, scores), "host and device entry points disagree"
        h2d = int(sum(p.pred.shape[0] * (48 + 3) + 8 for p in pairs))
        e2e = {"value": n * world / (em.item() / 1e3), "unit": "pairs/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": 104 * n}

    line = None
    if rank == 0:
        peak = ia.fp64_peak_tflops(local)
        flops = FLOP_PER_CELL * float(np.mean(cells)) + FLOP_PER_VISIT * float(np.mean(visits))
        k_ms = float(np.mean(kms))
        achieved = flops / (k_ms / 1e3) / 1e12 if k_ms > 0 else None
        roofline = {"kernel": "k_chain (NW chains: score matrix + NW + Kabsch + refine)",
                    "bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak if achieved else None, "traffic": None,
                    "peak_source": "measured FP64 FMA rate (indialign_fp64_peak) in this run",
                    "kernel_ms_per_step": k_ms, "kernel_share": k_ms / ms,
                    "nw_cells_per_step": int(np.mean(cells)),
                    "refine_visits_per_step": int(np.mean(visits)),
                    "warp_cycle_split": dict(zip(["nw_fill", "traceback", "detailed", "kabsch"],
                                                 [float(x) for x in np.mean(cyc, 0) / max(1.0, np.mean(cyc, 0).sum())]))}
        cpu = None
        if not args.no_cpu_baseline:
            r = cpu_baseline(pairs, args.cpu_sample)
            if r:
                cpu, sample, ref_s = r
                pos = {id(p): k for k, p in enumerate(pairs)}
                idx = [pos[id(p)] for p in sample]
                d = scores[idx] - ref_s
                cpu["parity_on_sample"] = {"min_dTM": float(d.min()), "max_abs_dTM": float(np.abs(d).max()),
                                           "pairs_below_ref_minus_1e-6": int(np.sum(d < -1e-6))}
        line = {"metric": METRIC, "value": value, "unit": "pairs/s", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": desc, "pairs_per_gpu": n, "mode": "plain",
                           "l2": "flushed by a 256 MB write before every step",
                           "parallelism": f"independent pairs per GPU x{world}"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": int(np.mean(launches)), "clocks": clocks,
                "stage_ms": dict(zip(["seeds", "seed_bank", "ss", "gapless", "local_fragment",
                                      "threading_dp", "dense_local_fragment", "topk", "dp_refine",
                                      "offset_dp", "weighted", "total"],
                                     [round(float(x), 2) for x in np.mean(stg, 0)])),
                "mean_tm": float(scores.mean())}
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
