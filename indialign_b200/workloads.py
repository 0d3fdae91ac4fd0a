"""Seeded synthetic RNA C1' trace pairs.

The reference ships no generator for its benchmark shapes; the public PDB and
competition datasets it was measured on need a network.  These generators
stand in for them with the shapes, sizes and value distributions of the five
workloads the search is measured on:

  single      L=64, sigma=2.0, all valid, lnorm=L                      (seed 0)
  batch4096   4096 pairs, L~U(40,300), sigma~U(0.5,14), 5 % invalid per mask
  hard1024    1024 pairs, L log-uniform 30..1500; half "hard": the native keeps
              30-60 % of the pred's stems, the rest regenerated, sigma~U(4,14)
  train200k   ranker training pairs, L 40..300 (generated lazily)
  learned16k  16384 pairs, L~U(40,1000), sigma~U(0.5,14)

A trace is a chain of A-form hairpin stems (C1' radius 8.9 A, rise 2.8 A/nt,
twist 32.7 deg, stem length U{6..12} base pairs) joined by self-avoiding random
walk loops (5.9 A steps, 3.5 A exclusion).  The native is the pred plus iid
Gaussian noise, then a uniformly random rotation and a translation U(-50,50)
per axis.  Masks are uint8 0/1; valid = pred_valid & native_valid.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

RADIUS = 8.9
RISE = 2.8
TWIST = math.radians(32.7)
LOOP_STEP = 5.9
EXCLUSION = 3.5
# azimuth offset of the paired strand: puts paired C1' atoms ~10.4 A apart,
# inside the [9, 12] A window the SS detector looks for.
PAIR_PHASE = math.radians(72.0)
PAIR_DZ = 1.2


@dataclass
class Pair:
    pred: np.ndarray          # (L, 3) float64
    native: np.ndarray        # (L, 3) float64
    valid: np.ndarray         # (L,) uint8
    pred_valid: np.ndarray    # (L,) uint8
    native_valid: np.ndarray  # (L,) uint8
    lnorm: float
    sigma: float = 0.0
    hard: bool = False


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    """Uniform rotation from a normalised Gaussian quaternion."""
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a*a + b*b - c*c - d*d, 2*(b*c - a*d), 2*(b*d + a*c)],
        [2*(b*c + a*d), a*a - b*b + c*c - d*d, 2*(c*d - a*b)],
        [2*(b*d - a*c), 2*(c*d + a*b), a*a - b*b - c*c + d*d],
    ])


def _hairpin(n_bp: int, rng: np.random.Generator) -> np.ndarray:
    """Local coordinates of one hairpin: 5' strand up the helix, a 4-nt loop
    over the top, 3' strand back down paired with the 5' strand."""
    k = np.arange(n_bp)
    ang = k * TWIST
    s5 = np.stack([RADIUS * np.cos(ang), RADIUS * np.sin(ang), k * RISE], 1)
    ang3 = ang + PAIR_PHASE
    s3 = np.stack([RADIUS * np.cos(ang3), RADIUS * np.sin(ang3),
                   k * RISE + PAIR_DZ], 1)[::-1]
    top_a, top_b = s5[-1], s3[0]
    mid = 0.5 * (top_a + top_b) + np.array([0.0, 0.0, 6.0])
    loop = []
    for f in (0.2, 0.4, 0.6, 0.8):  # quadratic arc over the top
        p = (1 - f) ** 2 * top_a + 2 * f * (1 - f) * mid + f * f * top_b
        loop.append(p)
    return np.concatenate([s5, np.array(loop), s3], 0)


def _walk(start: np.ndarray, direction: np.ndarray, n: int, placed: list,
          rng: np.random.Generator) -> np.ndarray:
    """Self-avoiding persistent random walk of n steps from start."""
    out = []
    pts = np.concatenate(placed, 0) if placed else np.zeros((0, 3))
    cur, d = start.copy(), direction / (np.linalg.norm(direction) + 1e-12)
    for _ in range(n):
        for _try in range(24):
            nd = d + rng.standard_normal(3) * 0.6
            nd /= np.linalg.norm(nd)
            cand = cur + nd * LOOP_STEP
            ok = True
            if pts.shape[0]:
                ok = np.min(np.sum((pts - cand) ** 2, 1)) >= EXCLUSION ** 2
            if ok and out:
                ok = np.min(np.sum((np.array(out) - cand) ** 2, 1)) >= EXCLUSION ** 2
            if ok:
                break
        out.append(cand)
        cur, d = cand, nd
    return np.array(out).reshape(-1, 3)


def make_trace(L: int, rng: np.random.Generator, return_stems: bool = False):
    """C1' trace of length L: alternating loops and hairpin stems."""
    placed: list = []
    segs: list = []   # (start, stop, is_stem)
    n = 0
    cur = np.zeros(3)
    d = rng.standard_normal(3)
    while n < L:
        loop_n = int(rng.integers(1, 6))
        loop_n = min(loop_n, L - n)
        if loop_n > 0:
            w = _walk(cur, d, loop_n, placed, rng)
            placed.append(w)
            segs.append((n, n + loop_n, False))
            n += loop_n
            cur = w[-1]
            if w.shape[0] >= 2:
                d = w[-1] - w[-2]
        if n >= L:
            break
        n_bp = int(rng.integers(6, 13))
        hp = _hairpin(n_bp, rng)
        take = min(hp.shape[0], L - n)
        R = random_rotation(rng)
        local = hp @ R.T
        shift = cur + d / (np.linalg.norm(d) + 1e-12) * LOOP_STEP - local[0]
        h = (local + shift)[:take]
        placed.append(h)
        segs.append((n, n + take, True))
        n += take
        cur = h[-1]
        d = h[-1] - h[-2] if take >= 2 else d
    x = np.concatenate(placed, 0)[:L]
    x = x - x.mean(0)
    return (x, segs) if return_stems else x


def _kabsch_np(P: np.ndarray, Q: np.ndarray):
    cp, cq = P.mean(0), Q.mean(0)
    H = (P - cp).T @ (Q - cq)
    U, _, Vt = np.linalg.svd(H)
    D = np.diag([1, 1, np.sign(np.linalg.det(Vt.T @ U.T))])
    R = Vt.T @ D @ U.T
    return R, cq - R @ cp


def make_pair(L: int, sigma: float, rng: np.random.Generator,
              invalid_frac: float = 0.0, hard: bool = False) -> Pair:
    pred, segs = make_trace(L, rng, return_stems=True)
    if hard:
        nat = make_trace(L, np.random.default_rng(rng.integers(1 << 62)))
        stems = [s for s in segs if s[2]]
        keep = rng.uniform(0.3, 0.6)
        for (a, b, _) in stems:
            if rng.uniform() < keep and b - a >= 3:
                R, t = _kabsch_np(pred[a:b], nat[a:b])
                nat[a:b] = pred[a:b] @ R.T + t
        base = nat
    else:
        base = pred
    native = base + rng.standard_normal((L, 3)) * sigma
    native = native @ random_rotation(rng).T + rng.uniform(-50, 50, 3)
    if invalid_frac > 0:
        pv = (rng.uniform(size=L) >= invalid_frac).astype(np.uint8)
        nv = (rng.uniform(size=L) >= invalid_frac).astype(np.uint8)
    else:
        pv = np.ones(L, np.uint8)
        nv = np.ones(L, np.uint8)
    return Pair(np.ascontiguousarray(pred), np.ascontiguousarray(native),
                (pv & nv).astype(np.uint8), pv, nv, float(L), sigma, hard)


def single(seed: int = 0) -> list[Pair]:
    """One L=64 pair, sigma 2.0, all valid."""
    rng = np.random.default_rng(seed)
    return [make_pair(64, 2.0, rng)]


def batch(n: int = 4096, lo: int = 40, hi: int = 300, seed: int = 1,
          invalid_frac: float = 0.05, sigma_lo: float = 0.5,
          sigma_hi: float = 14.0) -> list[Pair]:
    """n pairs, L~U(lo,hi), sigma~U(sigma_lo,sigma_hi), masks 5 % invalid."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        s = float(rng.uniform(sigma_lo, sigma_hi))
        out.append(make_pair(L, s, rng, invalid_frac))
    return out


def hard(n: int = 1024, seed: int = 2) -> list[Pair]:
    """Uneven batch, L log-uniform 30..1500, every other pair hard."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        L = int(round(math.exp(rng.uniform(math.log(30), math.log(1500)))))
        if i % 2 == 0:
            out.append(make_pair(L, float(rng.uniform(4, 14)), rng, 0.05, hard=True))
        else:
            out.append(make_pair(L, float(rng.uniform(0.5, 14)), rng, 0.05))
    return out


def learned(n: int = 16384, seed: int = 4) -> list[Pair]:
    """Learned-vs-plain workload: n pairs, L~U(40,1000), as batch()."""
    return batch(n, 40, 1000, seed)


def _batch_job(args):
    n, lo, hi, seed = args
    return batch(n, lo, hi, seed=seed)


def parallel_batch(n: int, lo: int, hi: int, seed: int, chunk: int = 256, procs: int = 8) -> list[Pair]:
    """batch()-distributed pairs generated in chunks by a spawn process pool
    (safe to start before or after CUDA initialisation); chunk c draws from
    seed * 100003 + c, so the result depends only on (n, lo, hi, seed, chunk)."""
    import multiprocessing as mp
    jobs = [(min(chunk, n - s), lo, hi, seed * 100003 + c) for c, s in enumerate(range(0, n, chunk))]
    if procs <= 1 or len(jobs) == 1:
        return [p for j in jobs for p in _batch_job(j)]
    with mp.get_context("spawn").Pool(min(procs, len(jobs))) as pool:
        return [p for part in pool.imap(_batch_job, jobs) for p in part]


def subsample(pairs: list[Pair], k: int, seed: int = 7) -> list[Pair]:
    """Fixed-seed subsample keeping the length distribution (sorted strata)."""
    if k >= len(pairs):
        return list(pairs)
    order = sorted(range(len(pairs)), key=lambda i: pairs[i].pred.shape[0])
    rng = np.random.default_rng(seed)
    strata = np.array_split(np.array(order), k)
    return [pairs[int(rng.choice(s))] for s in strata]
