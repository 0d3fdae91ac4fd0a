"""Golden fixtures for the parity tests, produced by the reference's own build.

Runs here, where the reference sources exist:

    make -C oracle && python tests/golden/make_golden.py          # small sets
    python tests/golden/make_golden.py shapes [cfg1] [cfg2]         # workload shapes

oracle/_ref/libindialign_ref.so is the reference's `make cpu` build compiled
from its sources (oracle/Makefile); ref_trace_search (oracle/ref_stages.cpp)
replays its stage order through the reference's own stage functions to record
the running best after every stage.  Outputs are small .npz files: the packed
inputs of each case group and the reference's results.

`shapes` writes the stratified samples of the two batch workloads the search
is quoted on (golden_cfg1.npz: 48 pairs of the 4096-pair shape, L 40-300,
5 % invalid per mask; golden_cfg2.npz: 18 pairs of the uneven hard shape,
L 30-1500, 10 of them hard, spread over every rescue stride branch of
rescue.h:30-46).  Every pair runs in its own single-threaded process
(OMP_NUM_THREADS=1, so the reference's inner loops take their serial,
deterministic path, as inside its batch entry); the longest hard pairs take
tens of minutes each.
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from indialign_b200 import abi, workloads as W  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(ROOT, "oracle", "_ref", "libindialign_ref.so")
STAGES = os.path.join(ROOT, "oracle", "_ref", "libindialign_ref_stages.so")
N_STAGES = 10


def pack(pairs):
    lens = [p.pred.shape[0] for p in pairs]
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    cat = lambda f, dt: np.concatenate([np.asarray(f(p), dt).reshape(-1) for p in pairs])
    return dict(off=off, pred=cat(lambda p: p.pred, np.float64),
                nat=cat(lambda p: p.native, np.float64), v=cat(lambda p: p.valid, np.uint8),
                pv=cat(lambda p: p.pred_valid, np.uint8), nv=cat(lambda p: p.native_valid, np.uint8),
                lnorm=np.array([p.lnorm for p in pairs], np.float64))


def run_ref(pairs):
    ref = abi.bind_reference_abi(ctypes.CDLL(REF))
    rc, s, R, t = abi.run_batch(ref, pairs)
    assert rc == 0
    st = ctypes.CDLL(STAGES)
    st.ref_trace_search.argtypes = [ctypes.POINTER(abi.NativePairInput),
                                    ctypes.POINTER(abi.NativeConfig),
                                    ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(abi.NativePairResult)]
    cfg = abi.default_config(ref)
    pk = abi.PackedInputs(pairs)
    trace = np.zeros((len(pairs), N_STAGES, 13))
    for k in range(len(pairs)):
        res = abi.NativePairResult()
        buf = np.zeros(N_STAGES * 13)
        st.ref_trace_search(ctypes.byref(pk.arr[k]), ctypes.byref(cfg),
                            buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(res))
        trace[k] = buf.reshape(N_STAGES, 13)
        assert abs(res.score - s[k]) < 1e-12, (k, res.score, s[k])
    return s, R, t, trace


def edge_pairs():
    rng = np.random.default_rng(77)
    out = []
    x = W.make_trace(40, rng)
    out.append(W.Pair(x.copy(), x.copy(), *(np.ones(40, np.uint8),) * 3, 40.0))  # identity
    p = W.make_pair(5, 1.0, rng)                                                  # tiny
    out.append(p)
    p = W.make_pair(30, 3.0, rng)
    p.lnorm = 2.0                                                                 # lnorm <= 2
    out.append(p)
    p = W.make_pair(24, 2.0, rng)
    p.valid = np.zeros(24, np.uint8)                                              # nothing valid
    out.append(p)
    p = W.make_pair(36, 4.0, rng, invalid_frac=0.2)
    p.valid = p.valid.copy()
    p.valid[p.valid == 1][:3] = 2
    idx = np.nonzero(p.valid)[0][:4]
    p.valid[idx] = 2                                                              # byte value 2
    out.append(p)
    out.append(W.make_pair(3, 0.5, rng))                                          # N = 3
    p = W.make_pair(50, 6.0, rng, invalid_frac=0.1)
    p.lnorm = float(p.valid.sum())                                                # lnorm = valid count
    out.append(p)
    p = W.make_pair(45, 2.0, rng)
    p.pred_valid = p.pred_valid.copy()
    p.pred_valid[10:20] = 0                                                       # one-sided gap
    p.valid = (p.pred_valid & p.native_valid).astype(np.uint8)
    out.append(p)
    return out


# (L, hard) of the uneven-shape sample: hard pairs whose valid counts fall in
# every stride bracket of local_jump (rescue.h:30-46: <=150, <=200, <=250,
# <=300, <=350, >350 residues) up to 1500, easy pairs spread log-uniformly
CFG2_SHAPES = [(60, True), (140, True), (190, True), (240, True), (290, True), (340, True),
               (420, True), (750, True), (1100, True), (1480, True),
               (30, False), (55, False), (120, False), (210, False), (330, False), (560, False),
               (900, False), (1350, False)]


def cfg1_pairs():
    """48 pairs stratified by length from 480 pairs of the 4096-pair shape."""
    return W.subsample(W.batch(480, 40, 300, seed=111), 48, seed=3)


def cfg2_pairs():
    rng = np.random.default_rng(222)
    out = []
    for L, hard in CFG2_SHAPES:
        sigma = float(rng.uniform(4, 14)) if hard else float(rng.uniform(0.5, 14))
        out.append(W.make_pair(L, sigma, rng, 0.05, hard=hard))
    return out


def _serial_init():
    os.environ["OMP_NUM_THREADS"] = "1"


def _ref_one(arg):
    """Reference batch entry and stage replay of one pair, single-threaded."""
    k, pair = arg
    s, R, t, trace = run_ref([pair])
    return k, s[0], R[0], t[0], trace[0]


def run_ref_serial(pairs, procs=8):
    """run_ref over `pairs`, one single-threaded process per pair, longest first."""
    import multiprocessing as mp
    order = sorted(range(len(pairs)), key=lambda i: -pairs[i].pred.shape[0])
    s = np.zeros(len(pairs))
    R = np.zeros((len(pairs), 9))
    t = np.zeros((len(pairs), 3))
    trace = np.zeros((len(pairs), N_STAGES, 13))
    with mp.get_context("spawn").Pool(procs, initializer=_serial_init) as pool:
        for k, sk, Rk, tk, trk in pool.imap_unordered(_ref_one, [(i, pairs[i]) for i in order]):
            s[k], R[k], t[k], trace[k] = sk, Rk, tk, trk
            print(f"  pair {k} L={pairs[k].pred.shape[0]} score={sk:.6f}", flush=True)
    return s, R, t, trace


def main_shapes(only=()):
    for name, pairs in (("cfg1", cfg1_pairs()), ("cfg2", cfg2_pairs())):
        if only and name not in only:
            continue
        s, R, t, trace = run_ref_serial(pairs)
        np.savez_compressed(os.path.join(OUT, f"golden_{name}.npz"), score=s, R=R, t=t, trace=trace,
                            sigma=np.array([p.sigma for p in pairs]),
                            hard=np.array([p.hard for p in pairs]), **pack(pairs))
        print(name, len(pairs), np.round(s, 4), flush=True)


def main():
    groups = {
        "single": W.single(0),
        "batch": [p for p in W.batch(64, seed=101) if p.pred.shape[0] <= 110][:12],
        "hard": [p for p in W.hard(48, seed=202) if p.pred.shape[0] <= 110][:4],
        "edge": edge_pairs(),
    }
    for name, pairs in groups.items():
        s, R, t, trace = run_ref(pairs)
        np.savez_compressed(os.path.join(OUT, f"golden_{name}.npz"), score=s, R=R, t=t,
                            trace=trace, sigma=np.array([p.sigma for p in pairs]), **pack(pairs))
        print(name, len(pairs), np.round(s, 4))
    # NW on explicit score matrices (nw_dp + nw_traceback), tie-heavy cases
    st = ctypes.CDLL(STAGES)
    st.ref_nw_align.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                ctypes.c_double, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    rng = np.random.default_rng(9)
    nw = {}
    # matrices are stored as uint16 grids q with score = q / 4096 (exact in
    # FP64); the large shapes only for the tie-heavy kinds, which compress
    shapes = [(1, 1), (1, 5), (5, 1), (3, 3), (7, 40), (64, 64), (65, 130), (130, 65),
              (200, 151), (300, 287)]
    kinds = ["uniform", "binary", "ss4", "cutoff"]
    case = 0
    for (np_, nn_) in shapes:
        for kind in kinds:
            if np_ * nn_ > 20000 and kind in ("uniform", "ss4"):
                continue
            gaps = (-0.6, 0.0, -1.0) if np_ * nn_ <= 20000 else ((-0.6,) if kind == "binary" else (0.0,))
            for gap in gaps:
                if kind == "uniform":
                    q = rng.integers(0, 4096, (np_, nn_))
                elif kind == "binary":
                    q = 4096 * (rng.uniform(size=(np_, nn_)) < 0.4)
                elif kind == "ss4":
                    q = rng.integers(0, 200, (np_, nn_)) + 2048 * (rng.uniform(size=(np_, nn_)) < 0.5)
                else:
                    d = rng.integers(0, 4096, (np_, nn_))
                    q = np.where(rng.uniform(size=(np_, nn_)) < 0.35, d, 0)
                q = q.astype(np.uint16)
                m = np.ascontiguousarray(q.astype(np.float64) / 4096.0)
                ap = np.zeros(min(np_, nn_), np.int32)
                an = np.zeros(min(np_, nn_), np.int32)
                na = st.ref_nw_align(m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), np_, nn_, gap,
                                     ap.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                     an.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
                nw[f"q{case}"] = q
                nw[f"g{case}"] = np.array([gap])
                nw[f"ap{case}"] = ap[:na].copy()
                nw[f"an{case}"] = an[:na].copy()
                case += 1
    np.savez_compressed(os.path.join(OUT, "golden_nw.npz"), **nw)
    print("nw cases", case)
    # std::sort tie order of the anchor candidates (count-only comparator)
    st = ctypes.CDLL(STAGES)
    rng = np.random.default_rng(5)
    rows = []
    for n in (1, 2, 5, 16, 17, 40, 100, 300, 1000):
        keys = rng.integers(3, 9, size=n).astype(np.int32)
        idx = np.arange(n, dtype=np.int32)
        k2, i2 = keys.copy(), idx.copy()
        st.ref_std_sort_desc(k2.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             i2.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n)
        rows.append((keys, i2))
    np.savez_compressed(os.path.join(OUT, "golden_sort.npz"),
                        **{f"keys{j}": r[0] for j, r in enumerate(rows)},
                        **{f"order{j}": r[1] for j, r in enumerate(rows)})


if __name__ == "__main__":
    if sys.argv[1:2] == ["shapes"]:
        main_shapes(tuple(sys.argv[2:]))
    else:
        main()
