"""Candidate ranker of the learned search: parameter blob, training on the
GPU through the library's BF16 tensor-core kernels, checkpoints, and the
shipped weights.

The network predicts, from 16 features of a candidate start of a refinement
loop -- a local-fragment or dense rescue window (indialign_c/rescue.h:50-117),
a threading-DP offset (rescue.h:121-190), a detailed-search fragment seed
(align.h:15-50) -- the score that refining it reaches.  It is an MLP
16 -> 128 -> 128 -> 1 with GELU, BF16 weights and activations, FP32
accumulation.  Training minimises mean squared error plus a pairwise
logistic ranking loss on row pairs drawn from the same candidate list, with
Adam.

Blob layout (FP32, INDIALIGN_RANKER_FLOATS): mean[16] std[16] W1[16][128]
b1[128] W2[128][128] b2[128] w3[128] b3, weights [in][out].
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import FEATURES, RANKER_FLOATS, IndialignError, load

HIDDEN = 128
MEAN = 0
STD = MEAN + FEATURES
W1 = STD + FEATURES
B1 = W1 + FEATURES * HIDDEN
W2 = B1 + HIDDEN
B2 = W2 + HIDDEN * HIDDEN
W3 = B2 + HIDDEN
B3 = W3 + HIDDEN
assert B3 + 1 == RANKER_FLOATS

WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ranker_weights.npy")


def default_weights() -> np.ndarray:
    """The shipped trained blob (trained by train_ranker.py on the GPU)."""
    if not os.path.exists(WEIGHTS_PATH):
        raise IndialignError(f"{WEIGHTS_PATH} missing: train with `python -m indialign_b200.train_ranker`")
    b = np.load(WEIGHTS_PATH)
    assert b.dtype == np.float32 and b.size == RANKER_FLOATS
    return np.ascontiguousarray(b)


def init_blob(mean: np.ndarray, std: np.ndarray, seed: int = 0) -> np.ndarray:
    """Random initial parameters (He-scaled weights, zero biases) with the
    given feature standardisation."""
    rng = np.random.default_rng(seed)
    b = np.zeros(RANKER_FLOATS, np.float32)
    b[MEAN:MEAN + FEATURES] = mean
    b[STD:STD + FEATURES] = np.where(std > 1e-6, std, 1.0)
    b[W1:B1] = rng.standard_normal(FEATURES * HIDDEN) * np.sqrt(2.0 / FEATURES)
    b[W2:B2] = rng.standard_normal(HIDDEN * HIDDEN) * np.sqrt(2.0 / HIDDEN)
    b[W3:B3] = rng.standard_normal(HIDDEN) * np.sqrt(1.0 / HIDDEN)
    return b


class Trainer:
    """Adam training of a blob on the GPU.  Device memory comes from torch
    (plumbing); every forward, loss, backward and update is one of the
    library's kernels."""

    def __init__(self, blob: np.ndarray, batch: int = 8192, lr: float = 1e-3, lam: float = 1.0,
                 beta1: float = 0.9, beta2: float = 0.999, eps: float = 1e-8):
        import torch
        self.torch = torch
        self.lib = load()
        dev = torch.device("cuda")
        self.batch, self.lr, self.lam = batch, lr, lam
        self.beta1, self.beta2, self.eps = beta1, beta2, eps
        self.blob = torch.tensor(np.asarray(blob, np.float32), device=dev)
        self.m = torch.zeros_like(self.blob)
        self.v = torch.zeros_like(self.blob)
        self.grad = torch.zeros_like(self.blob)
        u8 = torch.uint8
        self.packed = torch.empty(self.lib.indialign_mlp_packed_bytes(), dtype=u8, device=dev)
        self.save = torch.empty(self.lib.indialign_mlp_save_bytes(batch), dtype=u8, device=dev)
        self.work = torch.empty(self.lib.indialign_mlp_work_bytes(batch), dtype=u8, device=dev)
        self.y = torch.empty(batch, device=dev)
        self.dy = torch.empty(batch, device=dev)
        self.loss = torch.zeros(1, device=dev)
        self.steps = 0
        self.pack()

    @property
    def stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _ck(self, rc: int, what: str):
        if rc != 0:
            raise IndialignError(f"{what} rc={rc}: {self.lib.indialign_last_error().decode()}")

    def pack(self):
        self._ck(self.lib.indialign_mlp_pack(self.blob.data_ptr(), self.packed.data_ptr(), self.stream),
                 "mlp_pack")

    def forward(self, x, save: bool = False):
        """y = MLP(x) for x [n,16] float32 on the device (n <= batch with save)."""
        n = int(x.shape[0])
        assert x.dtype == self.torch.float32 and x.is_contiguous()
        y = self.y[:n] if save else self.torch.empty(n, device=x.device)
        sv = self.save.data_ptr() if save else None
        self._ck(self.lib.indialign_mlp_forward(self.packed.data_ptr(), x.data_ptr(), n, y.data_ptr(), sv,
                                                self.stream), "mlp_forward")
        return y

    def gradients(self, x, t):
        """Loss and gradient blob for one batch (rows (2i, 2i+1) paired)."""
        n = int(x.shape[0])
        assert n <= self.batch
        y = self.forward(x, save=True)
        self._ck(self.lib.indialign_mlp_loss(y.data_ptr(), t.data_ptr(), n, ctypes.c_float(self.lam),
                                             self.dy.data_ptr(), self.loss.data_ptr(), self.stream),
                 "mlp_loss")
        self._ck(self.lib.indialign_mlp_backward(self.packed.data_ptr(), self.dy.data_ptr(), n,
                                                 self.save.data_ptr(), self.grad.data_ptr(),
                                                 self.work.data_ptr(), self.stream), "mlp_backward")
        return self.loss, self.grad

    def step(self, x, t):
        loss, _ = self.gradients(x, t)
        self.steps += 1
        f = ctypes.c_float
        self._ck(self.lib.indialign_mlp_adam(self.blob.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                             self.v.data_ptr(), self.steps, f(self.lr), f(self.beta1),
                                             f(self.beta2), f(self.eps), self.stream), "mlp_adam")
        self.pack()
        return loss

    def predict(self, x, chunk: int = 1 << 20):
        out = []
        for s in range(0, int(x.shape[0]), chunk):
            out.append(self.forward(x[s:s + chunk].contiguous()))
        return self.torch.cat(out) if out else self.torch.empty(0, device=x.device)

    def numpy_blob(self) -> np.ndarray:
        return self.blob.detach().cpu().numpy().astype(np.float32)

    def checkpoint(self, path: str) -> None:
        """Save weights, Adam moments and step (resume with restore)."""
        cpu = lambda t: t.detach().cpu().numpy()
        save_checkpoint(path, cpu(self.blob), cpu(self.m), cpu(self.v), self.steps)

    def restore(self, path: str) -> None:
        blob, m, v, step = load_checkpoint(path)
        for dst, src in ((self.blob, blob), (self.m, m), (self.v, v)):
            dst.copy_(self.torch.from_numpy(src))
        self.steps = step
        self.pack()


CHECKPOINT_MAGIC = "indialign-ranker-v1"


def save_checkpoint(path: str, blob: np.ndarray, m: np.ndarray, v: np.ndarray, step: int) -> None:
    """Weights and Adam state in one .npz (header string, blob, moments, step)."""
    for a in (blob, m, v):
        assert np.asarray(a).size == RANKER_FLOATS
    np.savez(path, magic=np.array(CHECKPOINT_MAGIC), blob=np.asarray(blob, np.float32),
             m=np.asarray(m, np.float32), v=np.asarray(v, np.float32), step=np.array(int(step)))


def load_checkpoint(path: str):
    """(blob, m, v, step) from save_checkpoint."""
    z = np.load(path)
    if str(z["magic"]) != CHECKPOINT_MAGIC:
        raise IndialignError(f"{path}: not a ranker checkpoint")
    out = tuple(np.ascontiguousarray(z[k], np.float32) for k in ("blob", "m", "v"))
    if any(a.size != RANKER_FLOATS for a in out):
        raise IndialignError(f"{path}: wrong parameter count")
    return out + (int(z["step"]),)


def pair_rows(group: np.ndarray, rng: np.random.Generator) -> np.ndarray:
    """Random pairing of rows within each group: returns [m, 2] row indices,
    pairs in random order (odd leftovers of a group dropped)."""
    order = rng.permutation(group.size)
    order = order[np.argsort(group[order], kind="stable")]
    g = group[order]
    starts = np.r_[0, np.flatnonzero(g[1:] != g[:-1]) + 1]
    counts = np.diff(np.r_[starts, g.size])
    rank = np.arange(g.size) - np.repeat(starts, counts)
    keep = rank < np.repeat(counts // 2 * 2, counts)
    pairs = order[keep].reshape(-1, 2)
    return pairs[rng.permutation(pairs.shape[0])]


def train(feat: np.ndarray, label: np.ndarray, group: np.ndarray, epochs: int = 20, batch: int = 8192,
          lr: float = 1e-3, lam: float = 1.0, seed: int = 0, log=None) -> np.ndarray:
    """Train a blob on (feat, label) rows grouped by structure pair; returns
    the trained FP32 blob."""
    import torch
    mean = feat.mean(0).astype(np.float32)
    std = feat.std(0).astype(np.float32)
    tr = Trainer(init_blob(mean, std, seed), batch=batch, lr=lr, lam=lam)
    X = torch.tensor(feat, device="cuda")
    T = torch.tensor(label, device="cuda")
    rng = np.random.default_rng(seed + 1)
    half = batch // 2
    for ep in range(epochs):
        pairs = pair_rows(group, rng)
        idx_all = torch.tensor(pairs.reshape(-1), device="cuda")
        acc = torch.zeros(1, device="cuda")
        nb = 0
        for s in range(0, pairs.shape[0], half):
            idx = idx_all[2 * s:2 * (s + half)]
            acc += tr.step(X[idx].contiguous(), T[idx].contiguous())
            nb += 1
        if log:
            log(f"epoch {ep + 1}/{epochs}: {nb} steps, mean loss {float(acc.item()) / max(nb, 1):.5f}")
    return tr.numpy_blob()


def time_epoch(rows: int = 1 << 20, batch: int = 8192, groups: int = 4096, seed: int = 0,
               warmup: int = 3) -> dict:
    """Device time of one training epoch (the train() loop body: row gather,
    forward, loss, backward, Adam, repack) over `rows` synthetic feature rows
    in `groups` candidate lists, batch `batch`, after `warmup` untimed steps;
    plus the backward's share, timed with events around each backward call
    on the same stream."""
    import torch
    rng = np.random.default_rng(seed)
    feat = rng.standard_normal((rows, FEATURES)).astype(np.float32)
    label = rng.uniform(0.0, 1.0, rows).astype(np.float32)
    group = np.sort(rng.integers(0, groups, rows))
    tr = Trainer(init_blob(feat.mean(0), feat.std(0), seed), batch=batch)
    X = torch.tensor(feat, device="cuda")
    T = torch.tensor(label, device="cuda")
    pairs = pair_rows(group, rng)
    idx_all = torch.tensor(pairs.reshape(-1), device="cuda")
    half = batch // 2
    starts = list(range(0, pairs.shape[0] - half + 1, half))
    for s in starts[:warmup]:
        idx = idx_all[2 * s:2 * (s + half)]
        tr.step(X[idx].contiguous(), T[idx].contiguous())
    torch.cuda.synchronize()
    lib, st = tr.lib, tr.stream
    bw = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for s in starts:
        idx = idx_all[2 * s:2 * (s + half)]
        x, t = X[idx].contiguous(), T[idx].contiguous()
        n = int(x.shape[0])
        y = tr.forward(x, save=True)
        tr._ck(lib.indialign_mlp_loss(y.data_ptr(), t.data_ptr(), n, ctypes.c_float(tr.lam), tr.dy.data_ptr(),
                                      tr.loss.data_ptr(), st), "mlp_loss")
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record()
        tr._ck(lib.indialign_mlp_backward(tr.packed.data_ptr(), tr.dy.data_ptr(), n, tr.save.data_ptr(),
                                          tr.grad.data_ptr(), tr.work.data_ptr(), st), "mlp_backward")
        b1.record()
        bw.append((b0, b1))
        tr.steps += 1
        f = ctypes.c_float
        tr._ck(lib.indialign_mlp_adam(tr.blob.data_ptr(), tr.grad.data_ptr(), tr.m.data_ptr(), tr.v.data_ptr(),
                                      tr.steps, f(tr.lr), f(tr.beta1), f(tr.beta2), f(tr.eps), st), "mlp_adam")
        tr.pack()
    ev1.record()
    torch.cuda.synchronize()
    bw_ms = [a.elapsed_time(b) for a, b in bw]
    return {"rows": rows, "batch": batch, "steps": len(starts), "epoch_ms": ev0.elapsed_time(ev1),
            "backward_ms_per_step": float(np.mean(bw_ms)), "backward_ms_min": float(np.min(bw_ms)),
            "loss": float(tr.loss.item()), "grad_finite": bool(torch.isfinite(tr.grad).all().item())}
