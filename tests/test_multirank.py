"""The N>1 bench path on CPU: two gloo ranks shard the workload (each rank
its own batches of the same shape, no data-path collective) and combine
their times as the max over ranks."""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        batches, _ = bench.workload("batch24", 8, 3, rank)
        sig = np.array([b[0].pred[0, 0] for b in batches] + [len(b) for b in batches])
        my_ms = 10.0 + 5.0 * rank
        dist.barrier()
        mx = bench.reduce_max(dist, my_ms, "cpu")
        rate = bench.whole_job_rate(sum(len(b) for b in batches), world, mx)
        out.put((rank, sig.tolist(), mx, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_take_max_time():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    (r0, s0, m0, v0), (r1, s1, m1, v1) = res
    n = 3
    assert s0[n:] == s1[n:] == [8, 8, 8]          # same batch shapes on every rank
    assert s0[:n] != s1[:n]                          # different pairs per rank
    assert m0 == m1 == 15.0                          # max over ranks, agreed everywhere
    assert v0 == v1 == pytest.approx(2 * 24 / 0.015)


def test_shard_pairs_is_a_balanced_partition():
    import indialign_b200 as ia
    from indialign_b200 import workloads as W
    pairs = W.batch(40, 40, 600, seed=5)
    for k in (1, 2, 3, 8):
        sh = ia.shard_pairs(pairs, k)
        assert len(sh) == k
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(pairs)))
        cost = [sum(pairs[i].pred.shape[0] ** 3 for i in s) for s in sh]
        biggest = max(p.pred.shape[0] ** 3 for p in pairs)
        assert max(cost) - min(cost) <= biggest  # LPT: spread below one job
