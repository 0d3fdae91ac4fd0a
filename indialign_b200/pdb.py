"""C1' traces from PDB text, and search pairs of structures of unequal
length.

The search compares pred[i] with native[i] (same index); structures of
different lengths or with missing residues become one padded pair: residue
slots of the union of residue numbers, each side's missing slots marked
invalid in its own mask (pred_valid / native_valid), valid = both.  The
search's cross-index passes (NW, threading, local fragments) then find
offset correspondences, as for the reference's benchmark pairs
(benchmark/pdb_hard_benchmark.py:134-224: C1' extraction per model / chain,
pairing by residue number, lnorm = residues valid on both sides).
"""
from __future__ import annotations

import numpy as np

from .workloads import Pair


def _atom_c1(line: str):
    """(chain, xyz) of a C1' ATOM record, else None.  The residue number is
    not parsed here: the model and chain extractors of the reference
    benchmark never read it, so a blank or non-numeric resSeq (hybrid-36)
    must not stop them."""
    if not line.startswith("ATOM") or line[12:16].strip() != "C1'":
        return None
    xyz = (float(line[30:38]), float(line[38:46]), float(line[46:54]))
    return line[21], np.array(xyz, np.float64)


def c1_models(text: str) -> list[np.ndarray]:
    """C1' coordinates of every model closed by ENDMDL, in file order
    ([N, 3] each); a file without any closed model gives its C1' atoms as
    one model (benchmark/pdb_hard_benchmark.py:134-150: atoms after the last
    ENDMDL of a multi-model file are dropped)."""
    models, cur = [], []
    for line in text.splitlines():
        rec = line[:6].strip()
        if rec == "MODEL":
            cur = []
        elif rec == "ENDMDL":
            if cur:
                models.append(np.array(cur))
            cur = []
        else:
            a = _atom_c1(line)
            if a is not None:
                cur.append(a[1])
    if not models and cur:
        models.append(np.array(cur))
    return models


def c1_chains(text: str) -> dict[str, np.ndarray]:
    """{chain: C1' coordinates [N, 3] in file order} of the first model
    (benchmark/pdb_hard_benchmark.py:152-166)."""
    chains: dict[str, list] = {}
    for line in text.splitlines():
        if line[:6].strip() == "ENDMDL":
            break
        a = _atom_c1(line)
        if a is not None:
            chains.setdefault(a[0], []).append(a[1])
    return {ch: np.array(v) for ch, v in chains.items()}


def c1_by_chain(text: str) -> dict[str, dict[int, np.ndarray]]:
    """{chain: {residue number: C1' xyz}} of the first model; a repeated
    residue number keeps its last atom (benchmark/pdb_hard_benchmark.py:
    168-183)."""
    chains: dict[str, dict[int, np.ndarray]] = {}
    for line in text.splitlines():
        if line[:6].strip() == "ENDMDL":
            break
        a = _atom_c1(line)
        if a is not None:
            chains.setdefault(a[0], {})[int(line[22:26])] = a[1]
    return chains


def most_divergent_pair(models: list[np.ndarray]) -> tuple[int, int, float]:
    """(i, j, rmsd) of the two equal-length models with the largest C1' RMSD,
    the first such pair in scan order; ensembles of more than 20 models are
    scanned on model 0 and 19 models spread evenly over the rest
    (benchmark/pdb_hard_benchmark.py:195-207)."""
    n = len(models)
    idx = list(range(n))
    if n > 20:
        idx = [0] + [int(v) for v in np.linspace(1, n - 1, 19).astype(int)]
    best = (0, 1, -1.0)
    for a, i in enumerate(idx):
        for j in idx[a + 1:]:
            r = float(np.sqrt(np.mean(np.sum((models[i] - models[j]) ** 2, axis=1))))
            if r > best[2]:
                best = (i, j, r)
    return best


def pair_by_resnum(pred: dict[int, np.ndarray], native: dict[int, np.ndarray]) -> Pair:
    """One padded pair over the union of residue numbers (ascending)."""
    res = sorted(set(pred) | set(native))
    N = len(res)
    P = np.zeros((N, 3))
    Q = np.zeros((N, 3))
    pv = np.zeros(N, np.uint8)
    nv = np.zeros(N, np.uint8)
    for k, r in enumerate(res):
        if r in pred:
            P[k], pv[k] = pred[r], 1
        if r in native:
            Q[k], nv[k] = native[r], 1
    v = (pv & nv).astype(np.uint8)
    return Pair(P, Q, v, pv, nv, float(max(int(v.sum()), 1)), 0.0, False)


def ensemble_pair(text: str, min_len: int = 30, max_len: int = 4096):
    """(pair, (i, j, rmsd)) of an NMR-style ensemble's most divergent models,
    or None when it has fewer than two models, models of different lengths,
    or a length outside [min_len, max_len] (benchmark/pdb_hard_benchmark.py:
    257-272).  All residues valid, lnorm = length."""
    models = c1_models(text)
    if len(models) < 2 or len({len(m) for m in models}) != 1:
        return None
    n = len(models[0])
    if n < min_len or n > max_len:
        return None
    i, j, r = most_divergent_pair(models)
    ones = np.ones(n, np.uint8)
    return Pair(np.ascontiguousarray(models[i]), np.ascontiguousarray(models[j]), ones, ones.copy(),
                ones.copy(), float(n), 0.0, False), (i, j, r)


def longest_chain(text: str, min_len: int = 30):
    """(chain id, {residue number: xyz}) of the first model's longest chain
    (the first of equal length), or None below min_len residues."""
    chains = c1_by_chain(text)
    if not chains:
        return None
    best = max(chains, key=lambda c: len(chains[c]))
    return (best, chains[best]) if len(chains[best]) >= min_len else None


def family_pairs(texts: list[str], min_shared: int = 20, max_len: int = 4096) -> list[Pair]:
    """Structures of one family: the longest chain of the first structure is
    the native, the longest chain of each later one a prediction, paired by
    residue number; pairs with fewer than min_shared residues on both sides
    or more than max_len slots are left out (benchmark/pdb_hard_benchmark.py:
    355-385)."""
    chains = [c for c in (longest_chain(t) for t in texts) if c is not None]
    if len(chains) < 2:
        return []
    native = chains[0][1]
    out = []
    for _, pred in chains[1:]:
        p = pair_by_resnum(pred, native)
        if int(p.valid.sum()) < min_shared or len(p.valid) > max_len:
            continue
        out.append(p)
    return out


def pair_padded(pred: np.ndarray, native: np.ndarray, lnorm: float | None = None) -> Pair:
    """Two traces of possibly different lengths, without residue numbers:
    both padded to the longer one with invalid slots.  lnorm defaults to the
    native length (the reference structure's)."""
    Lp, Ln = len(pred), len(native)
    N = max(Lp, Ln)
    P = np.zeros((N, 3))
    Q = np.zeros((N, 3))
    P[:Lp], Q[:Ln] = pred, native
    pv = np.zeros(N, np.uint8)
    nv = np.zeros(N, np.uint8)
    pv[:Lp], nv[:Ln] = 1, 1
    v = (pv & nv).astype(np.uint8)
    return Pair(P, Q, v, pv, nv, float(lnorm if lnorm is not None else Ln), 0.0, False)


def c1_pdb_text(coords: np.ndarray, valid: np.ndarray | None = None, chain: str = "A",
                first_resnum: int = 1) -> str:
    """PDB ATOM records of a C1' trace (residues with valid == 0 left out)."""
    lines = []
    for i, (x, y, z) in enumerate(np.asarray(coords, np.float64)):
        if valid is not None and not valid[i]:
            continue
        r = first_resnum + i
        lines.append(f"ATOM  {len(lines) + 1:>5d}  C1'   A {chain}{r:>4d}    "
                     f"{x:>8.3f}{y:>8.3f}{z:>8.3f}  1.00  0.00           C")
    return "\n".join(lines) + "\nEND\n"
