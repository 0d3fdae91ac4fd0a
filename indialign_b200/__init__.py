"""indialign_b200: B200 (sm_100a) implementation of INDIalign's RNA TM-score
superposition search behind the reference's C ABI.

The product is libindialign.so (built from csrc/ by `make -C
indialign_b200/csrc`), exporting the reference's four entry points with its
struct layouts plus a batched entry point with options.  This module is the
ctypes shim the reference's own Python callers use, plus numpy helpers.  There
is no CPU path: when the library is missing or no CUDA device is usable the
calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Sequence

import numpy as np

from . import abi
from .abi import NativeConfig, NativePairInput, NativePairResult

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("INDIALIGN_B200_LIB", os.path.join(HERE, "libindialign.so"))
STAGES = 12
COUNTERS = 12
TRACE_STAGES = 10
KERNEL_MS = 6
MODE_PLAIN, MODE_LEARNED, MODE_COLLECT = 0, 1, 2
CAND_LOCAL, CAND_THREAD, CAND_DENSE, CAND_DET, CAND_MAIN = 0, 1, 2, 3, 4
CAND_KINDS = 5
RANK_LOCAL, RANK_THREAD, RANK_DENSE, RANK_DET_SS, RANK_DET_DP, RANK_MAIN = 1, 2, 4, 8, 16, 32
CAND_NAMES = ("local", "threading", "dense", "detailed", "seed_bank")
RANKER_FLOATS = 18849
RANK_STATS = 50
RANK_STAT_NAMES = ("gated", "fallback", "audit", "pruned", "windows", "refined",
                   "audit_miss", "small")
FEATURES = 16

_lib = None


class IndialignError(RuntimeError):
    pass


class BatchOptions(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_void_p), ("device", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("profile", ctypes.c_int),
                ("stage_ms", ctypes.POINTER(ctypes.c_double)),
                ("counters", ctypes.POINTER(ctypes.c_longlong)),
                ("kernel_ms", ctypes.POINTER(ctypes.c_double)),
                ("stage_best", ctypes.POINTER(ctypes.c_double)),
                ("mode", ctypes.c_int),
                ("ranker", ctypes.POINTER(ctypes.c_float)),
                ("top_k", ctypes.c_int),
                ("margin", ctypes.c_double),
                ("audit_rate", ctypes.c_double),
                ("seed", ctypes.c_ulonglong),
                ("rank_stats", ctypes.POINTER(ctypes.c_longlong)),
                ("win_feat", ctypes.POINTER(ctypes.c_float)),
                ("win_label", ctypes.POINTER(ctypes.c_float)),
                ("win_cap", ctypes.c_longlong),
                ("win_score", ctypes.POINTER(ctypes.c_float)),
                ("rank_mask", ctypes.c_int),
                ("rank_min_len", ctypes.c_int),
                ("win_select", ctypes.POINTER(ctypes.c_int))]


def build():
    """Compile the CUDA library in-tree (nvcc, sm_100a)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", os.path.join(HERE, "csrc"), "-j8"], check=True)


def load(path: str | None = None) -> ctypes.CDLL:
    """Load libindialign.so and bind its ABI; raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise IndialignError(
            f"{p} not found: build it with `make -C {os.path.join(HERE, 'csrc')}`")
    lib = abi.bind_reference_abi(ctypes.CDLL(p))
    lib.indialign_cuda_available.argtypes = []
    lib.indialign_cuda_available.restype = ctypes.c_int
    lib.indialign_tmscore_search_batch_ex.argtypes = [
        ctypes.c_int, ctypes.POINTER(NativePairInput), ctypes.POINTER(NativeConfig),
        ctypes.POINTER(BatchOptions), ctypes.POINTER(NativePairResult)]
    lib.indialign_tmscore_search_batch_ex.restype = ctypes.c_int
    lib.indialign_last_error.argtypes = []
    lib.indialign_last_error.restype = ctypes.c_char_p
    lib.indialign_inject_failure.argtypes = [ctypes.c_int]
    lib.indialign_inject_failure.restype = None
    lib.indialign_tmscore_search_device.argtypes = [
        ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
        ctypes.POINTER(ctypes.c_double), ctypes.POINTER(NativeConfig),
        ctypes.POINTER(BatchOptions), ctypes.c_void_p]
    lib.indialign_tmscore_search_device.restype = ctypes.c_int
    lib.indialign_tmscore_search_padded.argtypes = [
        ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p, ctypes.c_void_p,
        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
        ctypes.POINTER(NativeConfig), ctypes.POINTER(BatchOptions), ctypes.c_void_p]
    lib.indialign_tmscore_search_padded.restype = ctypes.c_int
    lib.indialign_fp64_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.indialign_fp64_peak.restype = ctypes.c_int
    lib.indialign_fp32_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.indialign_fp32_peak.restype = ctypes.c_int
    lib.indialign_candidate_count.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
    lib.indialign_candidate_count.restype = ctypes.c_int
    lib.indialign_get_tuning.argtypes = [ctypes.POINTER(ctypes.c_int)] * 3
    lib.indialign_get_tuning.restype = ctypes.c_int
    lib.indialign_set_tuning.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.indialign_set_tuning.restype = ctypes.c_int
    lib.indialign_pair_costs.argtypes = [ctypes.c_int, ctypes.POINTER(NativePairInput),
                                         ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.indialign_pair_costs.restype = ctypes.c_int
    lib.indialign_shard_pairs.argtypes = [ctypes.c_int, ctypes.POINTER(NativePairInput), ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int)]
    lib.indialign_shard_pairs.restype = ctypes.c_int
    lib.indialign_tmscore_search_multi.argtypes = [
        ctypes.c_int, ctypes.POINTER(NativePairInput), ctypes.POINTER(NativeConfig),
        ctypes.POINTER(BatchOptions), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
        ctypes.POINTER(NativePairResult)]
    lib.indialign_tmscore_search_multi.restype = ctypes.c_int
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    for name, args, res in (
            ("indialign_mlp_packed_bytes", [], sz),
            ("indialign_mlp_save_bytes", [ctypes.c_int], sz),
            ("indialign_mlp_work_bytes", [ctypes.c_int], sz),
            ("indialign_mlp_pack", [vp, vp, vp], ctypes.c_int),
            ("indialign_mlp_forward", [vp, vp, ctypes.c_int, vp, vp, vp], ctypes.c_int),
            ("indialign_mlp_loss", [vp, vp, ctypes.c_int, ctypes.c_float, vp, vp, vp], ctypes.c_int),
            ("indialign_mlp_backward", [vp, vp, ctypes.c_int, vp, vp, vp, vp], ctypes.c_int),
            ("indialign_gemm_bf16", [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int,
                                     vp], ctypes.c_int),
            ("indialign_mlp_adam", [vp, vp, vp, vp, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, vp], ctypes.c_int)):
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    if path is None:
        _lib = lib
    return lib


def default_config() -> NativeConfig:
    return abi.default_config(load())


def last_error() -> str:
    return load().indialign_last_error().decode()


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def learned_options(opts: BatchOptions, ranker: np.ndarray, top_k: int = 8, margin: float = 0.02,
                    audit_rate: float = 0.02, seed: int = 0,
                    rank_stats: np.ndarray | None = None, rank_mask: int = 0,
                    rank_min_len: int = 0) -> BatchOptions:
    """Fill the learned-mode fields of `opts` (keeps `ranker` referenced by
    the caller, which must outlive the call)."""
    assert ranker.dtype == np.float32 and ranker.size == RANKER_FLOATS and ranker.flags.c_contiguous
    opts.mode = MODE_LEARNED
    opts.ranker = _fptr(ranker)
    opts.top_k = int(top_k)
    opts.margin = float(margin)
    opts.audit_rate = float(audit_rate)
    opts.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    opts.rank_mask = int(rank_mask)
    opts.rank_min_len = int(rank_min_len)
    if rank_stats is not None:
        assert rank_stats.dtype == np.int64 and rank_stats.size >= RANK_STATS  # [5][10]
        opts.rank_stats = rank_stats.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    return opts


def candidate_count(plen: int, nlen: int, kind: int = 2) -> int:
    """Candidates of kind CAND_* of a pair with plen / nlen valid residues."""
    return int(load().indialign_candidate_count(int(plen), int(nlen), int(kind)))


def candidate_offsets(pairs: Sequence) -> np.ndarray:
    """[5, n+1] start of each pair's candidates per kind in the per-candidate
    arrays (kinds back to back): pair p of kind k at off[k, p]:off[k, p+1]
    (for CAND_DET the pair's two alignment slots of equal size)."""
    n = len(pairs)
    cnt = np.zeros((CAND_KINDS, n), np.int64)
    for i, p in enumerate(pairs):
        pl, nl = int(np.count_nonzero(p.pred_valid)), int(np.count_nonzero(p.native_valid))
        for k in range(CAND_KINDS):
            cnt[k, i] = candidate_count(pl, nl, k)
    off = np.zeros((CAND_KINDS, n + 1), np.int64)
    base = 0
    for k in range(CAND_KINDS):
        off[k, 0] = base
        off[k, 1:] = base + np.cumsum(cnt[k])
        base = int(off[k, -1])
    return off


def search(pairs: Sequence, cfg: NativeConfig | None = None, profile: bool = False,
           stage_ms: np.ndarray | None = None, counters: np.ndarray | None = None,
           stage_best: np.ndarray | None = None, kernel_ms: np.ndarray | None = None,
           stream: int | None = None, ranker: np.ndarray | None = None, top_k: int = 8,
           margin: float = 0.02, audit_rate: float = 0.02, seed: int = 0,
           rank_stats: np.ndarray | None = None):
    """Run the batched search on the GPU.

    pairs: objects with .pred/.native (L,3) float64, .valid/.pred_valid/
    .native_valid (L,) uint8 and .lnorm.  Returns (score[n], R[n,9], t[n,3]).
    With `ranker` (FP32 parameter blob) the dense local-fragment rescue runs
    in learned mode: top_k windows per pair, all windows when the predicted
    top-1 / top-k margin is below `margin` or on an audit draw.
    """
    lib = load()
    cfg = cfg or default_config()
    pk = abi.PackedInputs(pairs)
    res = (NativePairResult * max(1, pk.n))()
    opts = BatchOptions()
    opts.device = -1
    opts.profile = int(profile)
    if ranker is not None:
        learned_options(opts, ranker, top_k, margin, audit_rate, seed, rank_stats)
    if stage_ms is not None:
        assert stage_ms.dtype == np.float64 and stage_ms.size >= STAGES
        opts.stage_ms = stage_ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if counters is not None:
        assert counters.dtype == np.int64 and counters.size >= COUNTERS
        opts.counters = counters.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    if kernel_ms is not None:
        assert kernel_ms.dtype == np.float64 and kernel_ms.size >= KERNEL_MS
        opts.kernel_ms = kernel_ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if stream is not None:
        opts.stream = ctypes.c_void_p(stream)
    if stage_best is not None:
        assert stage_best.dtype == np.float64 and stage_best.size >= pk.n * TRACE_STAGES * 13
        opts.stage_best = stage_best.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg),
                                               ctypes.byref(opts), res)
    if rc != 0:
        raise IndialignError(f"indialign_tmscore_search_batch_ex rc={rc}: {last_error()}")
    return abi.results_to_numpy(res, pk.n)


RANK_ALL = RANK_LOCAL | RANK_THREAD | RANK_DENSE | RANK_DET_SS | RANK_DET_DP | RANK_MAIN


def collect_windows(pairs: Sequence, cfg: NativeConfig | None = None,
                    ranker: np.ndarray | None = None, rank_mask: int = RANK_ALL):
    """Plain search in COLLECT mode: every rescue candidate's 16 raw features
    and refined score.  Returns (results, feat[C,16] f32, label[C] f32 (NaN
    where the pair's pass did not run), off[5, n+1]) with pair p's candidates
    of kind k at off[k, p]:off[k, p+1].  With `ranker`, also the predicted
    scores: (results, feat, label, off, score).  rank_mask picks the lists
    recorded (default every kind)."""
    lib = load()
    cfg = cfg or default_config()
    pk = abi.PackedInputs(pairs)
    woff = candidate_offsets(pairs)
    W = int(woff[-1, -1])
    feat = np.zeros((max(W, 1), FEATURES), np.float32)
    label = np.zeros(max(W, 1), np.float32)
    res = (NativePairResult * max(1, pk.n))()
    opts = BatchOptions()
    opts.device = -1
    opts.mode = MODE_COLLECT
    opts.rank_mask = int(rank_mask)
    opts.win_feat = _fptr(feat)
    opts.win_label = _fptr(label)
    opts.win_cap = W
    score = None
    if ranker is not None:
        assert ranker.dtype == np.float32 and ranker.size == RANKER_FLOATS
        opts.ranker = _fptr(ranker)
        score = np.zeros(max(W, 1), np.float32)
        opts.win_score = _fptr(score)
    rc = lib.indialign_tmscore_search_batch_ex(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts), res)
    if rc != 0:
        raise IndialignError(f"indialign_tmscore_search_batch_ex(collect) rc={rc}: {last_error()}")
    out = (abi.results_to_numpy(res, pk.n), feat[:W], label[:W], woff)
    return out + (score[:W],) if ranker is not None else out


def search_tensors(pred, native, valid=None, pred_valid=None, native_valid=None, lengths=None,
                   lnorm=None, cfg: NativeConfig | None = None, ranker: np.ndarray | None = None,
                   top_k: int = 8, margin: float = 0.02, audit_rate: float = 0.02, seed: int = 0):
    """Search a padded batch of CUDA tensors, the (B, N, 3) shape of the
    reference's torch scorer: pred / native (B, N, 3), masks (B, N) (bool or
    uint8; pred_valid / native_valid default to valid, valid to all ones),
    lengths (B,) residues in use per row (default N), lnorm (B,) (default the
    lengths).  Runs on the current torch stream; returns torch tensors
    score (B,), R (B, 9), t (B, 3) on the device.  float64 contiguous inputs
    are read in place."""
    import torch
    lib = load()
    cfg = cfg or default_config()
    if pred.ndim != 3 or pred.shape != native.shape or pred.shape[2] != 3 or not pred.is_cuda:
        raise ValueError("pred and native must be matching (B, N, 3) CUDA tensors")
    B, N, _ = pred.shape
    dev = pred.device
    P = pred.to(torch.float64).contiguous()
    Q = native.to(torch.float64).contiguous()
    ones = torch.ones((B, N), dtype=torch.uint8, device=dev)
    V = ones if valid is None else valid.to(device=dev, dtype=torch.uint8).contiguous()
    PV = V if pred_valid is None else pred_valid.to(device=dev, dtype=torch.uint8).contiguous()
    NV = V if native_valid is None else native_valid.to(device=dev, dtype=torch.uint8).contiguous()
    lens = np.full(B, N, np.int32) if lengths is None else np.ascontiguousarray(
        torch.as_tensor(lengths).cpu().numpy(), np.int32)
    ln = lens.astype(np.float64) if lnorm is None else np.ascontiguousarray(
        torch.as_tensor(lnorm).cpu().numpy(), np.float64)
    out = torch.empty((B, 13), dtype=torch.float64, device=dev)
    opts = BatchOptions()
    opts.device = dev.index if dev.index is not None else -1
    opts.stream = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    if ranker is not None:
        learned_options(opts, ranker, top_k, margin, audit_rate, seed)
    rc = lib.indialign_tmscore_search_padded(
        B, N, lens.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), P.data_ptr(), Q.data_ptr(), V.data_ptr(),
        PV.data_ptr(), NV.data_ptr(), ln.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(cfg),
        ctypes.byref(opts), out.data_ptr())
    if rc != 0:
        raise IndialignError(f"indialign_tmscore_search_padded rc={rc}: {last_error()}")
    return out[:, 0], out[:, 1:10], out[:, 10:13]


TUNE_BUCKETS = 3
TUNE_FIELDS = ("max_len", "bank_chunk", "bank_cutoff_major", "chain_chunk", "chain_smem_trace")


def get_tuning() -> dict:
    """The kernel-shape table in use: {"split", "min_pairs", "rows": [dict per
    length bucket]} (indialign_get_tuning)."""
    lib = load()
    split, mp = ctypes.c_int(), ctypes.c_int()
    t = (ctypes.c_int * (TUNE_BUCKETS * len(TUNE_FIELDS)))()
    lib.indialign_get_tuning(ctypes.byref(split), ctypes.byref(mp), t)
    rows = [dict(zip(TUNE_FIELDS, t[b * len(TUNE_FIELDS):(b + 1) * len(TUNE_FIELDS)])) for b in range(TUNE_BUCKETS)]
    return {"split": split.value, "min_pairs": mp.value, "rows": rows}


def set_tuning(table: dict | None) -> None:
    """Replace the kernel-shape table for this process (None: reload it from
    its file), in get_tuning()'s form."""
    lib = load()
    if table is None:
        rc = lib.indialign_set_tuning(0, 0, None)
    else:
        flat = (ctypes.c_int * (TUNE_BUCKETS * len(TUNE_FIELDS)))(
            *[int(r[f]) for r in table["rows"] for f in TUNE_FIELDS])
        rc = lib.indialign_set_tuning(int(table["split"]), int(table["min_pairs"]), flat)
    if rc != 0:
        raise IndialignError(f"indialign_set_tuning rc={rc}: {last_error()}")


def write_tuning(table: dict, path: str, header: str = "") -> None:
    """Write a table in the library's file format (tune_b200.txt)."""
    with open(path, "w") as f:
        for line in header.splitlines():
            f.write(f"# {line}\n")
        f.write(f"split {int(table['split'])}\nmin_pairs {int(table['min_pairs'])}\n")
        for b, r in enumerate(table["rows"]):
            f.write(f"bucket {b} " + " ".join(f"{k} {int(r[k])}" for k in TUNE_FIELDS) + "\n")


def pair_costs(pairs: Sequence) -> tuple[np.ndarray, np.ndarray]:
    """(cost, tm0) per pair from the library's work estimate
    (indialign_pair_costs): NW-cell units, the rescue passes weighted by
    their likelihood judged from tm0, the TM-score under one Kabsch of all
    valid residues.  Host only."""
    lib = load()
    pk = abi.PackedInputs(list(pairs))
    cost = np.zeros(pk.n)
    tm0 = np.zeros(pk.n)
    rc = lib.indialign_pair_costs(pk.n, pk.arr, cost.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                  tm0.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    if rc != 0:
        raise IndialignError(f"indialign_pair_costs rc={rc}")
    return cost, tm0


def shard_pairs(pairs: Sequence, n_shards: int) -> list[list[int]]:
    """Work-balanced split of a batch over n_shards devices or ranks
    (indialign_shard_pairs: longest-processing-time greedy over
    pair_costs()).  Deterministic, so every rank computes the same split.
    Returns the pair indices of every shard, ascending."""
    n_shards = max(1, int(n_shards))
    lib = load()
    pk = abi.PackedInputs(list(pairs))
    shard = np.zeros(max(pk.n, 1), np.int32)
    rc = lib.indialign_shard_pairs(pk.n, pk.arr, n_shards, shard.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
    if rc != 0:
        raise IndialignError(f"indialign_shard_pairs rc={rc}")
    return [[i for i in range(pk.n) if shard[i] == k] for k in range(n_shards)]


def search_multi(pairs: Sequence, devices: Sequence[int], cfg: NativeConfig | None = None,
                 ranker: np.ndarray | None = None, rank_stats: np.ndarray | None = None, **learned):
    """Search a batch over several GPUs of this process through
    indialign_tmscore_search_multi: shard_pairs() split, one host thread and
    context per device, results in the batch's order.  No collective: pairs
    are independent."""
    lib = load()
    cfg = cfg or default_config()
    pk = abi.PackedInputs(list(pairs))
    res = (NativePairResult * max(pk.n, 1))()
    opts = BatchOptions()
    if ranker is not None:
        learned_options(opts, ranker, rank_stats=rank_stats, **learned)
    devs = np.ascontiguousarray(devices, np.int32)
    rc = lib.indialign_tmscore_search_multi(pk.n, pk.arr, ctypes.byref(cfg), ctypes.byref(opts),
                                            devs.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(devs), res)
    if rc != 0:
        raise IndialignError(f"indialign_tmscore_search_multi rc={rc}: {last_error()}")
    return abi.results_to_numpy(res, pk.n)


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput (TFLOP/s) of the device."""
    v = ctypes.c_double(0.0)
    rc = load().indialign_fp64_peak(device, ctypes.byref(v))
    if rc != 0:
        raise IndialignError(f"indialign_fp64_peak rc={rc}")
    return v.value


def fp32_peak_tflops(device: int = 0) -> float:
    """Measured FP32 FMA throughput (TFLOP/s) of the device."""
    v = ctypes.c_double(0.0)
    rc = load().indialign_fp32_peak(device, ctypes.byref(v))
    if rc != 0:
        raise IndialignError(f"indialign_fp32_peak rc={rc}")
    return v.value
