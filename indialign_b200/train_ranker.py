"""Train the rescue-candidate ranker on the GPU.

  python -m indialign_b200.train_ranker --pairs 200000 --heldout 20000 \
      --out indialign_b200/ranker_weights.npy

1. Synthetic training pairs (L ~ U(40, 300), sigma ~ U(0.5, 14) A, random
   rigid transform, 5 % invalid residues per mask) and held-out pairs from a
   different seed.
2. Labels: the plain GPU search in COLLECT mode records every rescue
   candidate's 16 features and refined score (local-fragment windows,
   threading-DP offsets, dense windows; pairs whose pass ran only).  Per pair
   and kind at most --per-pair candidates are kept: the best --keep-top by
   label plus a random draw of the rest.
3. Training: MSE + 10 x pairwise ranking loss (--lam), Adam (lr 1e-3, batch 8192,
   --epochs), every step on the library's BF16 tensor-core kernels.
4. Held-out evaluation: how often the top-k predicted windows contain the
   pair's best window score, and the margin-fallback rate.
"""
from __future__ import annotations

import argparse
import json
import sys
import time

import numpy as np


def generate(n: int, lo: int, hi: int, seed: int, procs: int = 8):
    from indialign_b200 import workloads as W
    return W.parallel_batch(n, lo, hi, seed, procs=procs)


def groups(off, kind: int, i: int):
    """Candidate ranges [a, b) of pair i's lists of one kind: one list, or
    the two alignment slots of the detailed searches."""
    import indialign_b200 as ia
    a, b = int(off[kind, i]), int(off[kind, i + 1])
    if kind != ia.CAND_DET:
        return [(a, b)]
    h = (b - a) // 2
    return [(a, a + h), (a + h, b)]


def collect(pairs, chunk: int, per_pair: int, keep_top: int, seed: int, log):
    """Features / labels / group ids of the kept candidates of every list
    whose pass ran; a group is one list (pair, kind, slot)."""
    import indialign_b200 as ia
    rng = np.random.default_rng(seed)
    F, Y, G = [], [], []
    t0 = time.time()
    for s in range(0, len(pairs), chunk):
        part = pairs[s:s + chunk]
        _, feat, label, off = ia.collect_windows(part)
        for kind in range(ia.CAND_KINDS):
            for i in range(len(part)):
                for slot, (a, b) in enumerate(groups(off, kind, i)):
                    lab = label[a:b]
                    idx = np.flatnonzero(np.isfinite(lab))
                    if idx.size < 2:
                        continue
                    if idx.size > per_pair:
                        top = idx[np.argsort(-lab[idx], kind="stable")[:keep_top]]
                        rest = np.setdiff1d(idx, top)
                        idx = np.concatenate([top, rng.choice(rest, per_pair - keep_top, replace=False)])
                    F.append(feat[a + idx])
                    Y.append(lab[idx])
                    G.append(np.full(idx.size, 8 * (s + i) + 2 * kind + slot, np.int64))
        log(f"collect {min(s + chunk, len(pairs))}/{len(pairs)} pairs, {sum(y.size for y in Y)} windows, "
            f"{time.time() - t0:.0f} s")
    if not F:
        return np.zeros((0, 16), np.float32), np.zeros(0, np.float32), np.zeros(0, np.int64)
    return np.concatenate(F), np.concatenate(Y).astype(np.float32), np.concatenate(G)


def evaluate(blob, pairs, chunk: int, ks=(1, 4, 8, 16), margin: float = 0.02, log=print,
             dump: str | None = None):
    """Per candidate kind: how often the top-k predicted candidates contain
    the best refined score (exactly, within 1e-4 and within 1e-3), and the
    fraction of candidates an 8-candidate selection with the margin fallback
    refines."""
    import indialign_b200 as ia
    res = {}
    acc = [dict(tot=0, fb=0, frac=[], hits={k: 0 for k in ks}, near={k: 0 for k in ks},
                near4={k: 0 for k in ks}) for _ in range(ia.CAND_KINDS)]
    dumps = []
    for s in range(0, len(pairs), chunk):
        part = pairs[s:s + chunk]
        _, feat, label, off, pred = ia.collect_windows(part, ranker=blob)
        for kind in range(ia.CAND_KINDS):
            a = acc[kind]
            for i, (ga, gb) in ((i, g) for i in range(len(part)) for g in groups(off, kind, i)):
                lab = label[ga:gb]
                fin = np.isfinite(lab)
                if not fin.any():
                    continue
                # a detailed-search slot holds its last search's seeds
                n_used = int(np.flatnonzero(fin).max()) + 1
                lab = np.where(fin, lab, -np.inf)[:n_used]
                pr = pred[ga:ga + n_used]
                order = np.lexsort((np.arange(lab.size), -pr))
                a["tot"] += 1
                for k in ks:
                    top = lab[order[:k]].max()
                    a["hits"][k] += top >= lab.max()
                    a["near"][k] += top >= lab.max() - 1e-3
                    a["near4"][k] += top >= lab.max() - 1e-4
                fb = lab.size > 8 and pr[order[0]] - pr[order[7]] < margin
                a["fb"] += fb
                a["frac"].append(1.0 if (fb or lab.size <= 8) else 8.0 / lab.size)
                if dump is not None and len(dumps) < 600:
                    dumps.append((kind, lab.astype(np.float32), pr.astype(np.float32)))
    for kind, a in enumerate(acc):
        r = {"pairs": a["tot"], "fallback_rate": a["fb"] / max(a["tot"], 1),
             "refined_fraction": float(np.mean(a["frac"])) if a["frac"] else 0.0}
        for k in ks:
            r[f"hit@{k}"] = a["hits"][k] / max(a["tot"], 1)
            r[f"near@{k}"] = a["near"][k] / max(a["tot"], 1)
            r[f"near1e-4@{k}"] = a["near4"][k] / max(a["tot"], 1)
        res[ia.CAND_NAMES[kind]] = r
    if dump is not None and dumps:
        np.savez_compressed(dump, kind=np.array([d[0] for d in dumps]),
                            **{f"lab{i}": d[1] for i, d in enumerate(dumps)},
                            **{f"pred{i}": d[2] for i, d in enumerate(dumps)})
    log(json.dumps(res))
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--pairs", type=int, default=200000)
    ap.add_argument("--heldout", type=int, default=20000)
    ap.add_argument("--lo", type=int, default=40)
    ap.add_argument("--hi", type=int, default=300)
    ap.add_argument("--eval-hi", type=int, default=300)
    ap.add_argument("--seed", type=int, default=31)
    ap.add_argument("--eval-seed", type=int, default=32)
    ap.add_argument("--per-pair", type=int, default=256)
    ap.add_argument("--keep-top", type=int, default=32)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--lam", type=float, default=10.0)
    ap.add_argument("--chunk", type=int, default=512)
    ap.add_argument("--procs", type=int, default=8)
    ap.add_argument("--out", default="ranker_weights.npy")
    ap.add_argument("--dump", default=None, help="npz of held-out labels / predictions")
    ap.add_argument("--data", default=None, help="npz cache of the collected training windows")
    ap.add_argument("--eval-only", default=None,
                    help="evaluate this weight blob (.npy; 'default': the shipped one) on the held-out pairs, "
                         "beside an untrained network of the same shape, and exit")
    ap.add_argument("--time-epoch", type=int, default=0, metavar="ROWS",
                    help="time one training epoch over ROWS synthetic feature rows at --batch, print JSON "
                         "and exit")
    a = ap.parse_args(argv)

    def log(msg):
        print(f"[train_ranker] {msg}", file=sys.stderr, flush=True)

    t0 = time.time()
    if a.time_epoch:
        from indialign_b200 import ranker
        print(json.dumps(ranker.time_epoch(rows=a.time_epoch, batch=a.batch, seed=a.seed)))
        return
    if a.eval_only:
        from indialign_b200 import ranker
        eval_pairs = generate(a.heldout, a.lo, a.eval_hi, a.eval_seed, procs=a.procs)
        log(f"generated {len(eval_pairs)} held-out pairs in {time.time() - t0:.0f} s")
        blob = ranker.default_weights() if a.eval_only == "default" else np.load(a.eval_only).astype(np.float32)
        out = {"trained": evaluate(blob, eval_pairs, a.chunk, log=log, dump=a.dump),
               "untrained": evaluate(ranker.init_blob(blob[ranker.MEAN:ranker.MEAN + ranker.FEATURES],
                                                       blob[ranker.STD:ranker.STD + ranker.FEATURES], a.seed),
                                     eval_pairs, a.chunk, log=log),
               "heldout_pairs": len(eval_pairs), "seconds": time.time() - t0}
        print(json.dumps(out))
        return

    train_pairs = generate(a.pairs, a.lo, a.hi, a.seed, procs=a.procs)
    eval_pairs = generate(a.heldout, a.lo, a.eval_hi, a.eval_seed, procs=a.procs)
    log(f"generated {len(train_pairs)} + {len(eval_pairs)} pairs in {time.time() - t0:.0f} s")
    from indialign_b200 import ranker
    F, Y, G = collect(train_pairs, a.chunk, a.per_pair, a.keep_top, a.seed, log)
    log(f"training candidates: {F.shape[0]} from {len(np.unique(G))} (pair, kind) groups")
    if a.data:
        np.savez_compressed(a.data, feat=F, label=Y, group=G)
    t1 = time.time()
    blob = ranker.train(F, Y, G, epochs=a.epochs, batch=a.batch, lr=a.lr, lam=a.lam, seed=a.seed, log=log)
    log(f"trained in {time.time() - t1:.0f} s")
    np.save(a.out, blob)
    res = evaluate(blob, eval_pairs, a.chunk, log=log, dump=a.dump)
    res.update({"train_candidates": int(F.shape[0]), "train_groups": int(len(np.unique(G))),
                "epochs": a.epochs, "seconds": time.time() - t0})
    print(json.dumps(res))


if __name__ == "__main__":
    main()
