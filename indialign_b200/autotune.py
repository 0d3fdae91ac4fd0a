"""Kernel-shape tuner for the length buckets of the batched search.

Every task of the batched search runs with its pair's length-bucket row
(N <= 128, <= 512, longer) of a kernel-shape table (indialign_set_tuning /
tune_b200.txt beside the library): seed-bank items per CTA chunk and their
order, NW chains per CTA chunk, NW traces in shared memory; the table also
says whether a batch that spans buckets runs as concurrent per-bucket
sub-batches.  This script times candidate rows on
seeded synthetic batches of each bucket (the batch shape of the workloads:
sigma ~ U(0.5,14) A, 5 % invalid residues per mask, random rigid transform)
with the learned search (the default ranker), one knob at a time from the
current row, keeps the fastest, then times a mixed-length batch of the
workload's call size (L 40-1000, 2048 pairs) with and without the split,
and writes the table and a log of every measurement.

    python -m indialign_b200.autotune --out indialign_b200/tune_b200.txt \\
        --log profiles/autotune_b200.md

Times are the wall time of one synchronous call (host packing included),
the minimum of --repeats calls after one warm-up call.
"""
from __future__ import annotations

import argparse
import copy
import time

from . import ranker
from . import workloads as W

BUCKET_RANGES = [(40, 128), (129, 512), (513, 1200)]
KNOBS = [("bank_chunk", (128, 256, 512)), ("bank_cutoff_major", (1, 0)), ("chain_chunk", (16, 8, 32)),
         ("chain_smem_trace", (1, 0))]


def _time_search(ia, pairs, blob, repeats):
    """Minimum time (ms) of one learned-search call over `pairs`: the call is
    synchronous, so its wall time covers every sub-batch of a split."""
    best = None
    for r in range(repeats + 1):
        t0 = time.perf_counter()
        ia.search(pairs, ranker=blob)
        ms = 1e3 * (time.perf_counter() - t0)
        if r > 0:
            best = ms if best is None else min(best, ms)
    return float(best)


def tune(pairs_per_bucket=512, repeats=2, seed=11, log=print, mixed_pairs=2048):
    import indialign_b200 as ia
    blob = ranker.default_weights()
    table = ia.get_tuning()
    base = copy.deepcopy(table)
    for b, (lo, hi) in enumerate(BUCKET_RANGES):
        pairs = W.parallel_batch(pairs_per_bucket, lo, hi, seed=seed + b)
        row = dict(table["rows"][b])
        t0 = time.time()

        def run(r):
            t = copy.deepcopy(table)
            t["rows"][b] = r
            ia.set_tuning(t)
            return _time_search(ia, pairs, blob, repeats)

        cur = run(row)
        log(f"bucket {b} (L {lo}-{hi}, {len(pairs)} pairs): start {row} -> {cur:.1f} ms")
        for knob, values in KNOBS:
            for v in values:
                if v == row[knob]:
                    continue
                cand = dict(row, **{knob: v})
                ms = run(cand)
                log(f"  {knob}={v}: {ms:.1f} ms" + ("  (kept)" if ms < cur else ""))
                if ms < cur:
                    cur, row = ms, cand
        table["rows"][b] = row
        log(f"bucket {b}: {row} -> {cur:.1f} ms ({time.time() - t0:.0f} s of tuning)")
    # the split itself, on a mixed batch of the learned workload's lengths and
    # call size
    mixed = W.parallel_batch(mixed_pairs, 40, 1000, seed=seed + 7)
    res = {}
    for split in (1, 0):
        t = copy.deepcopy(table)
        t["split"] = split
        ia.set_tuning(t)
        res[split] = _time_search(ia, mixed, blob, repeats)
        log(f"mixed batch (L 40-1000, {len(mixed)} pairs), split={split}: {res[split]:.1f} ms")
    table["split"] = 1 if res[1] <= res[0] else 0
    ia.set_tuning(base)
    return table


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=512, help="pairs per bucket")
    ap.add_argument("--mixed-pairs", type=int, default=2048, help="pairs of the mixed batch (split on/off)")
    ap.add_argument("--repeats", type=int, default=2)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--out", default=None, help="table file to write (tune_b200.txt format)")
    ap.add_argument("--log", default=None, help="markdown log of the measurements")
    a = ap.parse_args()
    import torch
    import indialign_b200 as ia
    lines = []

    def log(s):
        print(s, flush=True)
        lines.append(s)

    log(f"device: {torch.cuda.get_device_name(0)}")
    table = tune(a.pairs, a.repeats, a.seed, log, a.mixed_pairs)
    log(f"table: {table}")
    if a.out:
        ia.write_tuning(table, a.out, header="kernel shapes per length bucket, written by "
                                             "python -m indialign_b200.autotune")
    if a.log:
        with open(a.log, "w") as f:
            f.write("# Kernel-shape tuning of the length buckets\n\nCommand:\n\n```\npython -m "
                    f"indialign_b200.autotune --pairs {a.pairs} --mixed-pairs {a.mixed_pairs} "
                    f"--repeats {a.repeats} --seed {a.seed}"
                    + (f" --out {a.out}" if a.out else "") + f" --log {a.log}\n```\n\n"
                    "Learned search (shipped ranker), wall time per synchronous call, minimum of the repeats.\n\n```\n")
            f.write("\n".join(lines) + "\n```\n")


if __name__ == "__main__":
    main()
