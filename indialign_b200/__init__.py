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

_lib = None


class IndialignError(RuntimeError):
    pass


class BatchOptions(ctypes.Structure):
    _fields_ = [("stream", ctypes.c_void_p), ("device", ctypes.c_int),
                ("use_graph", ctypes.c_int), ("profile", ctypes.c_int),
                ("stage_ms", ctypes.POINTER(ctypes.c_double)),
                ("counters", ctypes.POINTER(ctypes.c_longlong)),
                ("kernel_ms", ctypes.POINTER(ctypes.c_double)),
                ("stage_best", ctypes.POINTER(ctypes.c_double))]


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
    lib.indialign_fp64_peak.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    lib.indialign_fp64_peak.restype = ctypes.c_int
    if path is None:
        _lib = lib
    return lib


def default_config() -> NativeConfig:
    return abi.default_config(load())


def last_error() -> str:
    return load().indialign_last_error().decode()


def search(pairs: Sequence, cfg: NativeConfig | None = None, profile: bool = False,
           stage_ms: np.ndarray | None = None, counters: np.ndarray | None = None,
           stage_best: np.ndarray | None = None, kernel_ms: np.ndarray | None = None,
           stream: int | None = None):
    """Run the batched search on the GPU.

    pairs: objects with .pred/.native (L,3) float64, .valid/.pred_valid/
    .native_valid (L,) uint8 and .lnorm.  Returns (score[n], R[n,9], t[n,3]).
    """
    lib = load()
    cfg = cfg or default_config()
    pk = abi.PackedInputs(pairs)
    res = (NativePairResult * max(1, pk.n))()
    opts = BatchOptions()
    opts.device = -1
    opts.profile = int(profile)
    if stage_ms is not None:
        assert stage_ms.dtype == np.float64 and stage_ms.size >= STAGES
        opts.stage_ms = stage_ms.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if counters is not None:
        assert counters.dtype == np.int64 and counters.size >= COUNTERS
        opts.counters = counters.ctypes.data_as(ctypes.POINTER(ctypes.c_longlong))
    if kernel_ms is not None:
        assert kernel_ms.dtype == np.float64 and kernel_ms.size >= 4
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


def fp64_peak_tflops(device: int = 0) -> float:
    """Measured FP64 FMA throughput (TFLOP/s) of the device."""
    v = ctypes.c_double(0.0)
    rc = load().indialign_fp64_peak(device, ctypes.byref(v))
    if rc != 0:
        raise IndialignError(f"indialign_fp64_peak rc={rc}")
    return v.value
