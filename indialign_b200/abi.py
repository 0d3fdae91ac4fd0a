"""ctypes mirror of the INDIalign C ABI.

The three structs are field-for-field the reference's (indialign_c/api.h:10-36;
x86-64 sizes 56 / 56 / 104 bytes), exactly as its own Python callers declare
them (tests/test_cpp_smoke.py:12-27, benchmark/fair_benchmark.py:26-41).  The
helpers here bind any library exporting that ABI: this package's
libindialign.so, or another build of the same interface.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

c_double_p = ctypes.POINTER(ctypes.c_double)
c_uint8_p = ctypes.POINTER(ctypes.c_uint8)


class NativeConfig(ctypes.Structure):
    _fields_ = [("backend_mode", ctypes.c_int), ("use_fragment_search", ctypes.c_int),
                ("max_iter", ctypes.c_int), ("dp_iter", ctypes.c_int),
                ("max_mem_gb", ctypes.c_double), ("request_cuda", ctypes.c_int),
                ("rescue_score_1", ctypes.c_double), ("rescue_score_2", ctypes.c_double),
                ("early_term_score", ctypes.c_double)]


class NativePairInput(ctypes.Structure):
    _fields_ = [("length", ctypes.c_int),
                ("pred_xyz", c_double_p), ("native_xyz", c_double_p),
                ("valid_mask", c_uint8_p), ("pred_valid_mask", c_uint8_p),
                ("native_valid_mask", c_uint8_p), ("lnorm", ctypes.c_double)]


class NativePairResult(ctypes.Structure):
    _fields_ = [("score", ctypes.c_double), ("R", ctypes.c_double * 9),
                ("t", ctypes.c_double * 3)]


assert ctypes.sizeof(NativeConfig) == 56
assert ctypes.sizeof(NativePairInput) == 56
assert ctypes.sizeof(NativePairResult) == 104


def bind_reference_abi(lib: ctypes.CDLL, prefix: str = "indialign_") -> ctypes.CDLL:
    """Set argtypes/restype of the four reference entry points on lib."""
    f = getattr(lib, prefix + "default_config")
    f.argtypes = [ctypes.POINTER(NativeConfig)]
    f.restype = None
    f = getattr(lib, prefix + "tmscore_search")
    f.argtypes = [ctypes.POINTER(NativePairInput), ctypes.POINTER(NativeConfig),
                  ctypes.POINTER(NativePairResult)]
    f.restype = ctypes.c_int
    f = getattr(lib, prefix + "tmscore_search_batch")
    f.argtypes = [ctypes.c_int, ctypes.POINTER(NativePairInput),
                  ctypes.POINTER(NativeConfig), ctypes.POINTER(NativePairResult)]
    f.restype = ctypes.c_int
    return lib


class PackedInputs:
    """Keeps the numpy buffers alive behind an array of NativePairInput."""

    def __init__(self, pairs: Sequence):
        self.bufs = []
        self.arr = (NativePairInput * max(1, len(pairs)))()
        for k, p in enumerate(pairs):
            pf = np.ascontiguousarray(np.asarray(p.pred, np.float64).reshape(-1))
            nf = np.ascontiguousarray(np.asarray(p.native, np.float64).reshape(-1))
            v = np.ascontiguousarray(p.valid, np.uint8)
            pv = np.ascontiguousarray(p.pred_valid, np.uint8)
            nv = np.ascontiguousarray(p.native_valid, np.uint8)
            self.bufs.append((pf, nf, v, pv, nv))
            a = self.arr[k]
            a.length = int(pf.shape[0] // 3)
            a.pred_xyz = pf.ctypes.data_as(c_double_p)
            a.native_xyz = nf.ctypes.data_as(c_double_p)
            a.valid_mask = v.ctypes.data_as(c_uint8_p)
            a.pred_valid_mask = pv.ctypes.data_as(c_uint8_p)
            a.native_valid_mask = nv.ctypes.data_as(c_uint8_p)
            a.lnorm = float(p.lnorm)
        self.n = len(pairs)


def results_to_numpy(res, n: int):
    """(score[n], R[n,9], t[n,3]) from a NativePairResult array."""
    buf = np.frombuffer(res, dtype=np.float64, count=13 * n).reshape(n, 13)
    return buf[:, 0].copy(), buf[:, 1:10].copy(), buf[:, 10:13].copy()


def default_config(lib: ctypes.CDLL, prefix: str = "indialign_") -> NativeConfig:
    cfg = NativeConfig()
    getattr(lib, prefix + "default_config")(ctypes.byref(cfg))
    return cfg


def run_batch(lib: ctypes.CDLL, pairs: Sequence, cfg: NativeConfig | None = None,
              prefix: str = "indialign_"):
    """Call <prefix>tmscore_search_batch; returns (rc, score, R, t)."""
    if cfg is None:
        cfg = default_config(lib, prefix)
    pk = PackedInputs(pairs)
    res = (NativePairResult * max(1, pk.n))()
    rc = getattr(lib, prefix + "tmscore_search_batch")(
        pk.n, pk.arr, ctypes.byref(cfg), res)
    s, R, t = results_to_numpy(res, pk.n)
    return rc, s, R, t
