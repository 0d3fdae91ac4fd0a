"""CPU restatement of the learned window ranker, used ONLY as test
infrastructure (tests/ import it as the checker; the product never does).

* candidates(): the candidate starts the ranker scores: local-fragment
  windows, normal and dense (indialign_c/rescue.h:12-46 local_frag_lengths /
  local_jump, :65-78 loop order), and threading-DP offsets (rescue.h:136-153)
  as the segment of their overlap.
* window_features(): the 16 features of a candidate segment, FP64.
* mlp_forward() / mlp_backward() / loss(): the 16 -> 128 -> 128 -> 1 GELU
  MLP with the device's rounding points emulated (BF16 round-to-nearest-even
  of the standardised inputs, the hidden activations and the backward's
  pre-activation gradients; every product and sum in FP64 here).
* select(): top-k by (score desc, window asc), the margin fallback and the
  audit draw.
* adam(): one bias-corrected Adam step.

The reference has no learned component: parity of this part is pinned by
the FP64 finite-difference check of mlp_backward (tests/test_ranker.py) and
by the window schedule, which restates the reference loop and is checked
against the library's own count.  The schedule functions it is built from
(local_frag_lengths, local_jump, frag_lengths, start_positions) and the
detailed-search seed list are checked against the reference's own functions
(tests/test_oracle_stages.py).
"""
from __future__ import annotations

import numpy as np

FEATURES, HIDDEN = 16, 128
MEAN = 0
STD = 16
W1 = 32
B1 = W1 + FEATURES * HIDDEN
W2 = B1 + HIDDEN
B2 = W2 + HIDDEN * HIDDEN
W3 = B2 + HIDDEN
B3 = W3 + HIDDEN
SIZE = B3 + 1
GELU_C = 0.7978845608028654
GELU_A = 0.044715


# ---- window schedule (rescue.h:12-46, 65-78) -------------------------------
def local_frag_lengths(plen: int, nlen: int, dense: bool) -> list[int]:
    ml = min(plen, nlen)
    if ml < 4:
        return []
    out: list[int] = []
    if dense:
        for v in (ml, min(100, ml // 2), min(32, ml), min(24, ml), min(20, ml // 3), 16, 12, 8, 4):
            if v >= 4 and v not in out:
                out.append(v)
    else:
        a, b = min(20, ml // 3), min(100, ml // 2)
        if a >= 4:
            out.append(a)
        if b >= 4 and b != a:
            out.append(b)
    return out


def local_jump(length: int, dense: bool) -> int:
    if dense:
        j = 50 if length > 350 else 30 if length > 300 else 10 if length > 200 else 5
        return max(1, min(j, max(1, length // 4)))
    j = 45 if length > 250 else 35 if length > 200 else 25 if length > 150 else 15
    return max(1, min(j, max(1, length // 3)))


def thread_offsets(plen: int, nlen: int) -> list[tuple[int, int, int]]:
    """(overlap, ps, ns) of the threading-DP offsets (rescue.h:136-153)."""
    if min(plen, nlen) < 3:
        return []
    step = max(1, min(plen, nlen) // 50)
    out = []
    for off in range(-(nlen - 3), plen - 2, step):
        ps, ns = max(off, 0), max(-off, 0)
        out.append((min(plen - ps, nlen - ns), ps, ns))
    return out


def frag_lengths(L: int) -> list[int]:
    """fragment_lengths (seeds.h:15-22): {L, L/2, L/4, L/8, 64, 32, 16, 8, 4}
    within [4, L], distinct, descending."""
    out = []
    for v in (L, L // 2, L // 4, L // 8, 64, 32, 16, 8, 4):
        if 4 <= v <= L and v not in out:
            out.append(v)
    return sorted(out, reverse=True)


def start_positions(n: int, frag: int, ms: int) -> list[int]:
    """start_positions (seeds.h:24-37)."""
    total = n - frag + 1
    if total <= 0:
        return []
    if total <= ms:
        return list(range(total))
    step = max(1, total // ms)
    out = list(range(0, total, step))
    if out[-1] != total - 1:
        out.append(total - 1)
    return out


def det_seeds(na: int, ms: int = 50) -> list[tuple[int, int, int]]:
    """Seeds of a detailed search on na aligned points (align.h:33-37):
    the whole set, then windows (len, s, s)."""
    if na < 3:
        return []
    out = [(na, 0, 0)]
    for f in frag_lengths(na):
        out += [(f, s, s) for s in start_positions(na, f, ms)]
    return out


def candidates(plen: int, nlen: int, kind: int) -> list[tuple[int, int, int]]:
    """Kind 0 local windows, 1 threading offsets, 2 dense windows, 3
    detailed-search seeds (plen == nlen == aligned count)."""
    if kind == 3:
        return det_seeds(min(plen, nlen))
    return thread_offsets(plen, nlen) if kind == 1 else windows(plen, nlen, kind == 2)


def windows(plen: int, nlen: int, dense: bool = True) -> list[tuple[int, int, int]]:
    """(flen, ps, ns) in the reference's work order."""
    jp, jn = local_jump(plen, dense), local_jump(nlen, dense)
    out = []
    for flen in local_frag_lengths(plen, nlen, dense):
        plim, nlim = plen - flen + 1, nlen - flen + 1
        if plim <= 0 or nlim <= 0:
            continue
        for ps in range(0, plim, jp):
            for ns in range(0, nlim, jn):
                out.append((flen, ps, ns))
    return out


# ---- features ----------------------------------------------------------------
def kabsch(P: np.ndarray, Q: np.ndarray):
    """Least-squares rigid fit q ~ R p + t (SVD form)."""
    cp, cq = P.mean(0), Q.mean(0)
    H = (P - cp).T @ (Q - cq)
    U, _, Vt = np.linalg.svd(H)
    d = np.sign(np.linalg.det(Vt.T @ U.T))
    R = Vt.T @ np.diag([1.0, 1.0, d]) @ U.T
    return R, cq - R @ cp


def window_features(Pc: np.ndarray, Qc: np.ndarray, ssp: str, ssn: str, d0: float, lnorm: float,
                    best: float, win: tuple[int, int, int], kind: int) -> np.ndarray:
    """Features of candidate segment (flen, ps, ns) of kind `kind` on compact
    coordinates Pc [plen,3], Qc [nlen,3] and compact SS labels ('L' loop,
    '<' / '>' stem)."""
    flen, ps, ns = win
    plen, nlen = Pc.shape[0], Qc.shape[0]
    ml = min(plen, nlen)
    R, t = kabsch(Pc[ps:ps + flen], Qc[ns:ns + flen])

    def d2(P, Q):
        return (((P @ R.T + t) - Q) ** 2).sum(1)

    dw = d2(Pc[ps:ps + flen], Qc[ns:ns + flen])
    d0sq = d0 * d0
    s = ns - ps
    lo, hi = max(0, -s), min(plen, nlen - s)
    dd = d2(Pc[lo:hi], Qc[lo + s:hi + s]) if hi > lo else np.zeros(0)
    d00 = d2(Pc[:ml], Qc[:ml])
    rmsd = np.sqrt(dw.sum() / flen)
    stem_p = sum(c != "L" for c in ssp[ps:ps + flen]) / flen
    stem_n = sum(c != "L" for c in ssn[ns:ns + flen]) / flen
    f = [flen / ml, ps / max(1, plen - 1), ns / max(1, nlen - 1), s / ml, rmsd / 10.0,
         (1.0 / (1.0 + dd / d0sq)).sum() / lnorm, (dd < d0sq).sum() / ml, (dd < 4 * d0sq).sum() / ml,
         (1.0 / (1.0 + dw / d0sq)).sum() / flen, stem_p, stem_n, np.log(ml) / 7.0, best, 0.5 * kind,
         min(rmsd / d0, 10.0) / 10.0, (1.0 / (1.0 + d00 / d0sq)).sum() / lnorm]
    return np.array(f, np.float64)


# ---- MLP -----------------------------------------------------------------------
def bf16(x) -> np.ndarray:
    """Round FP32 values to BF16 (nearest, ties to even), returned as FP32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def gelu(x):
    return 0.5 * x * (1.0 + np.tanh(GELU_C * (x + GELU_A * x ** 3)))


def gelu_grad(x):
    th = np.tanh(GELU_C * (x + GELU_A * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * GELU_C * (1.0 + 3.0 * GELU_A * x * x)


def unpack(blob: np.ndarray):
    b = np.asarray(blob)
    if b.dtype != np.float64:
        b = b.astype(np.float32)
    return dict(mean=b[MEAN:MEAN + 16], std=b[STD:STD + 16], W1=b[W1:B1].reshape(16, 128),
                b1=b[B1:W2], W2=b[W2:B2].reshape(128, 128), b2=b[B2:W3], w3=b[W3:B3], b3=b[B3])


def mlp_forward(blob: np.ndarray, x: np.ndarray, emulate: bool = True):
    """Returns y and the activations.  emulate=True applies the device's BF16
    rounding points; False is the plain FP64 network on BF16 weights."""
    p = unpack(blob)
    r = bf16 if emulate else (lambda v: np.asarray(v, np.float64))
    mean, std = p["mean"].astype(np.float32), p["std"].astype(np.float32)
    inv = np.where(std > 0, np.float32(1.0) / std, np.float32(1.0)).astype(np.float32)
    xn = r((np.asarray(x, np.float32) - mean) * inv).astype(np.float64)
    W1b, W2b = bf16(p["W1"]).astype(np.float64), bf16(p["W2"]).astype(np.float64)
    z1 = xn @ W1b + p["b1"].astype(np.float64)
    h1 = r(gelu(z1).astype(np.float32) if emulate else gelu(z1)).astype(np.float64)
    z2 = h1 @ W2b + p["b2"].astype(np.float64)
    y = gelu(z2) @ p["w3"].astype(np.float64) + float(p["b3"])
    return y, dict(xn=xn, z1=z1, h1=h1, z2=z2, W1b=W1b, W2b=W2b, p=p)


def loss(y: np.ndarray, t: np.ndarray, lam: float):
    """MSE + lam x mean logistic ranking loss over row pairs (2i, 2i+1)."""
    y = np.asarray(y, np.float64)
    t = np.asarray(t, np.float64)
    n, m = y.size, y.size // 2
    L = ((y - t) ** 2).sum() / n
    dy = 2.0 * (y - t) / n
    for i in range(m):
        a, b = 2 * i, 2 * i + 1
        dt = t[a] - t[b]
        if abs(dt) > 1e-6:
            s = 1.0 if dt > 0 else -1.0
            z = -s * (y[a] - y[b])
            L += lam * (z if z > 20 else np.log1p(np.exp(z))) / m
            sig = 1.0 / (1.0 + np.exp(-z))
            dy[a] += -lam * s * sig / m
            dy[b] += lam * s * sig / m
    return L, dy


def mlp_backward(blob: np.ndarray, x: np.ndarray, dy: np.ndarray, emulate: bool = True) -> np.ndarray:
    """Gradient of sum(dy * y) w.r.t. the blob (mean/std entries zero)."""
    _, a = mlp_forward(blob, x, emulate)
    p = a["p"]
    r = (lambda v: bf16(np.asarray(v, np.float32)).astype(np.float64)) if emulate else (lambda v: v)
    dy = np.asarray(dy, np.float64)
    g = np.zeros(SIZE, np.float64)
    gz2 = dy[:, None] * p["w3"].astype(np.float64)[None, :] * gelu_grad(a["z2"])
    g[W3:B3] = (dy[:, None] * gelu(a["z2"])).sum(0)
    g[B3] = dy.sum()
    g[B2:W3] = gz2.sum(0)
    dz2 = r(gz2)
    g[W2:B2] = (a["h1"].T @ dz2).reshape(-1)
    dh1 = dz2 @ a["W2b"].T
    gz1 = dh1 * gelu_grad(a["z1"])
    g[B1:W2] = gz1.sum(0)
    dz1 = r(gz1)
    g[W1:B1] = (a["xn"].T @ dz1).reshape(-1)
    return g


def adam(w, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step on entries W1.. (mean/std untouched); returns new (w, m, v)."""
    w, m, v = (np.array(a, np.float64) for a in (w, m, v))
    g = np.asarray(g, np.float64)
    s = slice(W1, SIZE)
    m[s] = b1 * m[s] + (1 - b1) * g[s]
    v[s] = b2 * v[s] + (1 - b2) * g[s] ** 2
    w[s] -= lr * (m[s] / (1 - b1 ** step)) / (np.sqrt(v[s] / (1 - b2 ** step)) + eps)
    return w, m, v


# ---- selection ---------------------------------------------------------------------
MASK64 = (1 << 64) - 1


def mix64(z: int) -> int:
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def audit_draw(seed: int, p: int) -> float:
    return (mix64((seed ^ mix64((p + 0x9E3779B97F4A7C15) & MASK64)) & MASK64) >> 11) / 9007199254740992.0


def select(score: np.ndarray, k: int, margin: float, audit_rate: float, seed: int, p: int):
    """(count, windows ascending) of one gated pair: count -2 audit, -1 all
    (margin fallback or at most k windows), else k."""
    s = np.asarray(score, np.float32).copy()
    s[np.isnan(s)] = -np.inf
    W = s.size
    if W <= k:
        return -1, []
    order = sorted(range(W), key=lambda w: (-s[w], w))[:k]
    top1, topk = s[order[0]], s[order[-1]]
    lst = sorted(order)
    if audit_draw(seed, p) < audit_rate:
        return -2, lst
    if float(np.float32(top1 - topk)) < np.float32(margin):
        return -1, lst
    return k, lst


# ---- main seed-bank seeds ------------------------------------------------------
def main_seed_features(P: np.ndarray, Q: np.ndarray, valid: np.ndarray, sel: np.ndarray, anchor: bool,
                       d0: float, d0s: float, lnorm: float) -> np.ndarray:
    """Features of one main seed-bank seed (seeds.h:41-283) given its
    selection (seed & valid) on the full pair, FP64."""
    v = np.asarray(valid) != 0
    s = (np.asarray(sel) != 0) & v
    cnt = int(s.sum())
    if cnt >= 3:
        R, t = kabsch(P[s], Q[s])
    else:
        R, t = np.eye(3), np.zeros(3)
    d2 = (((P @ R.T + t) - Q) ** 2).sum(1)
    d0sq = d0 * d0
    term = 1.0 / (1.0 + d2 / d0sq)
    N = P.shape[0]
    vc = max(int(v.sum()), 1)
    idx = np.flatnonzero(s)
    first, span = (idx[0], idx[-1] - idx[0] + 1) if idx.size else (0, 0)
    rmsd = np.sqrt(d2[s].sum() / max(cnt, 1))
    f = [cnt / vc, first / max(N, 1), span / max(N, 1), 1.0 if anchor else 0.0, rmsd / 10.0,
         term[v].sum() / lnorm, (d2[v] < d0sq).sum() / vc, (d2[v] < 4 * d0sq).sum() / vc,
         term[s].sum() / max(cnt, 1), (d2[v] < d0s * d0s).sum() / vc, 0.0, np.log(max(N, 1)) / 7.0, 0.0,
         2.0, min(rmsd / d0, 10.0) / 10.0, term[s].sum() / lnorm]
    return np.array(f, np.float64)
