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
    cost, _ = ia.pair_costs(pairs)
    for k in (1, 2, 3, 8):
        sh = ia.shard_pairs(pairs, k)
        assert len(sh) == k
        flat = sorted(i for s in sh for i in s)
        assert flat == list(range(len(pairs)))
        load = [sum(cost[i] for i in s) for s in sh]
        assert max(load) - min(load) <= cost.max()  # LPT: spread below one job


def _kabsch_tm(p):
    """Same-index TM-score (no d8) under the SVD Kabsch of all valid residues."""
    v = p.valid != 0
    P, Q = p.pred[v], p.native[v]
    cp, cq = P.mean(0), Q.mean(0)
    U, _, Vt = np.linalg.svd((P - cp).T @ (Q - cq))
    D = np.diag([1, 1, np.sign(np.linalg.det(Vt.T @ U.T))])
    R = Vt.T @ D @ U.T
    d2 = (((P - cp) @ R.T + cq - Q) ** 2).sum(1)
    L = p.pred.shape[0]
    d0 = max(0.6 * np.sqrt(L - 0.5) - 2.5, 0.3) if L >= 30 else 0.3
    return (1 / (1 + d2 / d0 ** 2)).sum() / max(p.lnorm, 1.0)


def test_pair_cost_prior_and_rescue_weight():
    """tm0 is the TM-score of the global Kabsch superposition; at equal length
    a noisy pair (rescue passes likely) costs more than a close one."""
    import indialign_b200 as ia
    from indialign_b200 import workloads as W
    rng = np.random.default_rng(8)
    pairs = [W.make_pair(L, s, rng, 0.05) for L in (60, 200, 450) for s in (0.5, 14.0)]
    cost, tm0 = ia.pair_costs(pairs)
    ref = np.array([_kabsch_tm(p) for p in pairs])
    np.testing.assert_allclose(tm0, ref, atol=1e-6)
    for k in range(0, len(pairs), 2):
        assert tm0[k] > 0.5 and tm0[k + 1] < 0.3
        assert cost[k + 1] > 2 * cost[k]
    assert cost[-1] > cost[1]  # longer costs more


def test_search_multi_rejects_per_pair_outputs_and_fails_without_device():
    import ctypes
    import indialign_b200 as ia
    from indialign_b200 import abi, workloads as W
    lib = ia.load()
    pairs = W.batch(3, 40, 60, seed=2)
    pk = abi.PackedInputs(pairs)
    res = (ia.NativePairResult * 3)()
    devs = np.zeros(2, np.int32)
    opts = ia.BatchOptions()
    buf = np.zeros(3 * ia.TRACE_STAGES * 13)
    opts.stage_best = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    cfg = ia.default_config()
    rc = lib.indialign_tmscore_search_multi(3, pk.arr, ctypes.byref(cfg), ctypes.byref(opts),
                                            devs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 2, res)
    assert rc == -4 and "per-device" in ia.last_error()
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if not has_gpu:
        rc = lib.indialign_tmscore_search_multi(3, pk.arr, ctypes.byref(cfg), None,
                                                devs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), 2, res)
        assert rc == -2 and "device" in ia.last_error()


def _shard_rank_main(rank, world, port, out):
    """Each rank takes its shard of one batch (the same deterministic split on
    every rank), searches it with the oracle and gathers the results."""
    import ctypes
    import torch.distributed as dist
    import indialign_b200 as ia
    from indialign_b200 import abi, workloads as W
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), OMP_NUM_THREADS="1")
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pairs = W.batch(10, 40, 90, seed=17)
        shards = ia.shard_pairs(pairs, world)
        mine = shards[rank]
        ora = abi.bind_reference_abi(ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so")), prefix="ora_")
        _, s, _, _ = abi.run_batch(ora, [pairs[i] for i in mine], prefix="ora_")
        got = [None] * world
        dist.all_gather_object(got, (rank, mine, [float(x) for x in s], shards))
        out.put(got)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_search_their_shards_of_one_batch(oracle):
    """The multi-rank form of the split: every rank computes the same shards,
    searches its own, and the gathered scores equal one search of the whole
    batch."""
    import multiprocessing as mp
    from indialign_b200 import abi, workloads as W
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got = res[0]
    assert res[0] == res[1]
    assert got[0][3] == got[1][3]  # identical split on both ranks
    pairs = W.batch(10, 40, 90, seed=17)
    _, s_all, _, _ = abi.run_batch(oracle, pairs, prefix="ora_")
    s = np.zeros(len(pairs))
    for _, idx, sc, _ in got:
        s[idx] = sc
    assert sorted(i for _, idx, _, _ in got for i in idx) == list(range(len(pairs)))
    np.testing.assert_array_equal(s, s_all)
