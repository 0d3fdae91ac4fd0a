"""Accuracy comparison under a common scorer (the reference's
benchmark/fair_benchmark.py): every tool's (R, t) is scored by the same
formula with the same d0, so differences in the tools' own scoring conventions
drop out.

* `common_tm`: sum over all residues of 1 / (1 + d^2 / d0^2) after moving pred
  by (R, t), divided by lnorm -- no d8 cutoff (fair_benchmark.py:57-61);
  `common_tm_masked` counts only residues valid on both sides and divides by
  their number (pdb_hard_benchmark.py:114-120), the form `compare` uses, so
  padded PDB pairs (`pdb.ensemble_pair`, `pdb.family_pairs`) compare too.
* `d0_rna`: the RNA d0 both tools use (fair_benchmark.py:48-55).
* USalign (`run_usalign`): C1' PDB files in, `-atom " C1'" -TMscore 1 -m
  <file>` (sequence-dependent superposition), the second "TM-score=" of its
  output (normalised by the native) and the rotation file parsed
  (fair_benchmark.py:85-113).  No USalign binary ships with this package;
  pass its path to `compare` / `--usalign`.
* `compare`: this library's batched search on all pairs at once, USalign per
  pair when given, then wins / ties at 1e-6, deltas, a sign test and a
  Wilcoxon test, and strata by mean common TM (fair_benchmark.py:160-232).

Rotation conventions: this library returns R with aligned_d = sum_k p_k
R[3k+d] (indialign_c/core.h:127-132); `matrix_from_result` gives the matrix M
with aligned = M p + t, the form `common_tm` and USalign use.
"""
from __future__ import annotations

import argparse
import math
import os
import re
import subprocess
import tempfile
import time
from dataclasses import dataclass, field

import numpy as np

from . import pdb
from .workloads import Pair, random_rotation


def d0_rna(L: float) -> float:
    """RNA d0 of a structure of L residues (piecewise below 30)."""
    if L <= 11:
        return 0.3
    if L <= 15:
        return 0.4
    if L <= 19:
        return 0.5
    if L <= 23:
        return 0.6
    if L < 30:
        return 0.7
    return 0.6 * math.sqrt(L - 0.5) - 2.5


def common_tm(pred: np.ndarray, native: np.ndarray, M: np.ndarray, t: np.ndarray, d0: float,
              lnorm: float) -> float:
    """TM-score of pred moved by aligned = M p + t against native, every
    residue counted, no distance cutoff."""
    moved = pred @ np.asarray(M).T + np.asarray(t)
    d2 = np.sum((moved - native) ** 2, axis=1)
    return float(np.sum(1.0 / (1.0 + d2 / (d0 * d0))) / lnorm)


def common_tm_masked(pred: np.ndarray, native: np.ndarray, valid: np.ndarray, M: np.ndarray, t: np.ndarray,
                     d0: float) -> float:
    """common_tm over the residues valid on both sides, normalised by their
    count (benchmark/pdb_hard_benchmark.py:114-120); 0 when none is."""
    v = np.asarray(valid) != 0
    if not v.any():
        return 0.0
    moved = pred @ np.asarray(M).T + np.asarray(t)
    d2 = np.sum((moved - native) ** 2, axis=1)
    return float(np.sum(v / (1.0 + d2 / (d0 * d0))) / v.sum())


def matrix_from_result(R9: np.ndarray) -> np.ndarray:
    """This library's 9-double R (aligned_d = sum_k p_k R[3k+d]) as M with
    aligned = M p."""
    return np.asarray(R9, np.float64).reshape(3, 3).T


def random_walk_trace(n: int, rng: np.random.Generator) -> np.ndarray:
    """A C1'-like chain: a persistent random walk (unit direction nudged by
    N(0, 0.3^2) per axis each step, step length N(5.9, 0.5^2) A), centred."""
    x = np.zeros((n, 3))
    d = rng.standard_normal(3)
    d /= np.linalg.norm(d)
    for i in range(1, n):
        d = d + rng.standard_normal(3) * 0.3
        d /= np.linalg.norm(d)
        x[i] = x[i - 1] + d * (5.9 + rng.standard_normal() * 0.5)
    return x - x.mean(0)


def fair_pairs(n: int, seed: int = 42, lo: int = 40, hi: int = 300) -> list[Pair]:
    """The comparison's workload: native a random walk of L ~ U(lo, hi)
    residues, pred = a random rotation of it + N(0, sigma^2) noise per
    coordinate (sigma ~ U(0.5, 14)) + a N(0, 20^2) offset; all residues
    valid, lnorm = L."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L = int(rng.integers(lo, hi + 1))
        sigma = float(rng.uniform(0.5, 14.0))
        native = random_walk_trace(L, rng)
        pred = native @ random_rotation(rng).T + rng.standard_normal((L, 3)) * sigma + rng.standard_normal(3) * 20
        ones = np.ones(L, np.uint8)
        out.append(Pair(np.ascontiguousarray(pred), np.ascontiguousarray(native), ones, ones.copy(), ones.copy(),
                        float(L), sigma, False))
    return out


# ---- USalign ---------------------------------------------------------------

_TM_RE = re.compile(r"TM-score=\s+([\d.]+)")


def parse_usalign_scores(stdout: str) -> float:
    """The second reported TM-score (normalised by the second structure, the
    native), 0.0 when absent."""
    found = _TM_RE.findall(stdout)
    return float(found[1]) if len(found) >= 2 else 0.0


def parse_usalign_matrix(text: str) -> tuple[np.ndarray, np.ndarray]:
    """(M, t) from a rotation file: rows "m t[m] u[m][0] u[m][1] u[m][2]" for
    m = 0, 1, 2 (aligned = M p + t)."""
    M = np.zeros((3, 3))
    t = np.zeros(3)
    for line in text.splitlines():
        f = line.split()
        if len(f) == 5 and f[0] in ("0", "1", "2"):
            m = int(f[0])
            t[m] = float(f[1])
            M[m] = [float(v) for v in f[2:]]
    return M, t


def run_usalign(pred: np.ndarray, native: np.ndarray, usalign: str, timeout: float = 30.0,
                pred_valid: np.ndarray | None = None, native_valid: np.ndarray | None = None):
    """(score, M, t, seconds) of one USalign run on C1' traces (residues
    invalid on a side are left out of that side's file, with their residue
    numbers kept)."""
    with tempfile.TemporaryDirectory() as d:
        pp, pn, pm = (os.path.join(d, f) for f in ("pred.pdb", "native.pdb", "matrix.txt"))
        for path, xyz, v in ((pp, pred, pred_valid), (pn, native, native_valid)):
            with open(path, "w") as f:
                f.write(pdb.c1_pdb_text(xyz, v))
        t0 = time.perf_counter()
        out = subprocess.run([usalign, pp, pn, "-atom", " C1'", "-TMscore", "1", "-m", pm],
                             capture_output=True, text=True, timeout=timeout)
        dt = time.perf_counter() - t0
        M, t = parse_usalign_matrix(open(pm).read()) if os.path.exists(pm) else (np.eye(3), np.zeros(3))
    return parse_usalign_scores(out.stdout), M, t, dt


# ---- comparison ------------------------------------------------------------

STRATA = ((0.0, 0.17, "very hard (TM<0.17)"), (0.17, 0.3, "hard (0.17-0.3)"), (0.3, 0.5, "medium (0.3-0.5)"),
          (0.5, 0.7, "moderate (0.5-0.7)"), (0.7, 1.01, "easy (TM>0.7)"))


@dataclass
class Report:
    self_ours: np.ndarray
    common_ours: np.ndarray
    seconds_ours: float
    self_usalign: np.ndarray | None = None
    common_usalign: np.ndarray | None = None
    seconds_usalign: np.ndarray | None = None
    stats: dict = field(default_factory=dict)


def _stats(ci: np.ndarray, cu: np.ndarray) -> dict:
    d = ci - cu
    wins = int(np.sum(d > 1e-6))
    losses = int(np.sum(d < -1e-6))
    s = {"pairs": int(d.size), "wins": wins, "losses": losses, "ties": int(d.size) - wins - losses,
         "mean_delta": float(d.mean()), "median_delta": float(np.median(d)), "max_delta": float(d.max()),
         "min_delta": float(d.min())}
    nontie = d[np.abs(d) > 1e-6]
    if wins + losses > 0:
        from scipy.stats import binomtest
        s["sign_test_p"] = float(binomtest(wins, wins + losses, 0.5, alternative="greater").pvalue)
    if nontie.size >= 10:
        from scipy.stats import wilcoxon
        s["wilcoxon_p"] = float(wilcoxon(nontie, zero_method="wilcox", alternative="greater").pvalue)
    avg = (ci + cu) / 2
    strata = []
    for lo, hi, name in STRATA:
        m = (avg >= lo) & (avg < hi)
        if m.any():
            dm = d[m]
            strata.append({"stratum": name, "pairs": int(m.sum()), "wins": int(np.sum(dm > 1e-6)),
                           "losses": int(np.sum(dm < -1e-6)), "mean_delta": float(dm.mean())})
    s["strata"] = strata
    return s


def compare(pairs: list[Pair], usalign: str | None = None, search=None) -> Report:
    """Score this library's results (and USalign's, with its path) under the
    common scorer.  `search(pairs) -> (score, R9, t)` defaults to the batched
    GPU search."""
    if search is None:
        from . import search as search_fn
        search = search_fn
    t0 = time.perf_counter()
    s, R, t = search(pairs)
    secs = time.perf_counter() - t0

    def common(p, M, tt):  # residues valid on both sides, d0 of their count
        n = int(np.sum(p.valid != 0))
        return common_tm_masked(p.pred, p.native, p.valid, M, tt, d0_rna(max(n, 1)))

    rep = Report(np.asarray(s), np.array([common(p, matrix_from_result(R[k]), t[k]) for k, p in enumerate(pairs)]),
                 secs)
    if usalign:
        su, cu, du = [], [], []
        for p in pairs:
            sc, M, tu, dt = run_usalign(p.pred, p.native, usalign, pred_valid=p.pred_valid,
                                        native_valid=p.native_valid)
            su.append(sc)
            cu.append(common(p, M, tu))
            du.append(dt)
        rep.self_usalign, rep.common_usalign, rep.seconds_usalign = np.array(su), np.array(cu), np.array(du)
        rep.stats = _stats(rep.common_ours, rep.common_usalign)
    return rep


def format_report(rep: Report) -> str:
    n = rep.common_ours.size
    lines = [f"pairs: {n}",
             f"this library: mean common TM {rep.common_ours.mean():.6f}, mean self-reported "
             f"{rep.self_ours.mean():.6f}, max |self - common| "
             f"{np.max(np.abs(rep.self_ours - rep.common_ours)):.2e}, {rep.seconds_ours:.2f} s for the batch"]
    if rep.common_usalign is None:
        lines.append("USalign: not run (no binary given)")
        return "\n".join(lines)
    s = rep.stats
    lines += [f"USalign: mean common TM {rep.common_usalign.mean():.6f}, mean self-reported "
              f"{rep.self_usalign.mean():.6f}, {rep.seconds_usalign.mean() * 1e3:.1f} ms per pair",
              f"wins {s['wins']}  losses {s['losses']}  ties {s['ties']} (at 1e-6)",
              f"delta (this - USalign): mean {s['mean_delta']:+.6f} median {s['median_delta']:+.6f} "
              f"max {s['max_delta']:+.6f} min {s['min_delta']:+.6f}"]
    if "sign_test_p" in s:
        lines.append(f"sign test p = {s['sign_test_p']:.3e}")
    if "wilcoxon_p" in s:
        lines.append(f"Wilcoxon p = {s['wilcoxon_p']:.3e}")
    for st in s["strata"]:
        lines.append(f"  {st['stratum']:<22s} {st['pairs']:5d} pairs  wins {st['wins']:4d}  losses "
                     f"{st['losses']:4d}  mean delta {st['mean_delta']:+.6f}")
    return "\n".join(lines)


def pdb_pairs(ensembles: list[str], family: list[str]) -> list[Pair]:
    """Pairs from local PDB files: each ensemble file's most divergent model
    pair, and a family's later structures against its first."""
    out = []
    for path in ensembles:
        r = pdb.ensemble_pair(open(path).read())
        if r is not None:
            out.append(r[0])
    if family:
        out += pdb.family_pairs([open(p).read() for p in family])
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--pairs", type=int, default=50, help="synthetic random-walk pairs (without PDB input)")
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--usalign", default=None, help="path of a USalign binary")
    ap.add_argument("--pdb-ensemble", nargs="*", default=[], help="multi-model PDB files")
    ap.add_argument("--pdb-family", nargs="*", default=[], help="PDB files of one family (first = native)")
    a = ap.parse_args()
    pairs = pdb_pairs(a.pdb_ensemble, a.pdb_family) if (a.pdb_ensemble or a.pdb_family) \
        else fair_pairs(a.pairs, a.seed)
    if not pairs:
        raise SystemExit("no pairs")
    print(format_report(compare(pairs, a.usalign)))


if __name__ == "__main__":
    main()
