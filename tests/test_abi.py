"""The C-ABI library: loads, exports every symbol declared in include/*.h,
keeps the reference struct layouts and its host-side error behaviour.  No
device work is launched here."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import LIB_SO, ROOT
import indialign_b200 as ia
from indialign_b200 import abi, workloads as W


def _declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"\b(indialign_\w+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB_SO), "build with make -C indialign_b200/csrc"
    lib = ctypes.CDLL(LIB_SO)
    syms = _declared_symbols()
    assert {"indialign_default_config", "indialign_tmscore_search",
            "indialign_tmscore_search_batch", "indialign_cuda_available"} <= set(syms)
    for s in syms:
        assert hasattr(lib, s), s


def test_struct_sizes_match_reference_layout():
    assert ctypes.sizeof(abi.NativeConfig) == 56
    assert ctypes.sizeof(abi.NativePairInput) == 56
    assert ctypes.sizeof(abi.NativePairResult) == 104


def test_default_config_matches_reference():
    c = ia.default_config()
    assert (c.backend_mode, c.use_fragment_search, c.max_iter, c.dp_iter) == (0, 1, 20, 1)
    assert (c.max_mem_gb, c.request_cuda) == (20.0, 0)
    assert (c.rescue_score_1, c.rescue_score_2, c.early_term_score) == (0.5, 0.3, 0.99)


def test_default_config_equals_reference_build(ref):
    a, b = ia.default_config(), abi.default_config(ref)
    assert bytes(a) == bytes(b)


def test_length_nonpositive_returns_minus_one_and_leaves_output():
    lib = ia.load()
    inp = abi.NativePairInput()
    inp.length = 0
    cfg = ia.default_config()
    out = abi.NativePairResult()
    out.score = 3.25
    assert lib.indialign_tmscore_search(ctypes.byref(inp), ctypes.byref(cfg), ctypes.byref(out)) == -1
    assert out.score == 3.25


def test_batch_skips_nonpositive_lengths_without_device():
    # all pairs empty: nothing to do, rc 0, outputs untouched (reference
    # batch ignores the per-pair -1)
    lib = ia.load()
    arr = (abi.NativePairInput * 2)()
    arr[0].length = 0
    arr[1].length = -3
    res = (abi.NativePairResult * 2)()
    res[0].score = res[1].score = 9.0
    cfg = ia.default_config()
    assert lib.indialign_tmscore_search_batch(2, arr, ctypes.byref(cfg), res) == 0
    assert res[0].score == res[1].score == 9.0


def test_injected_failure_reports_code_and_writes_nothing():
    lib = ia.load()
    p = W.single(0)
    pk = abi.PackedInputs(p)
    res = (abi.NativePairResult * 1)()
    res[0].score = 5.0
    cfg = ia.default_config()
    lib.indialign_inject_failure(1)
    rc = lib.indialign_tmscore_search_batch(1, pk.arr, ctypes.byref(cfg), res)
    assert rc == -6
    assert res[0].score == 5.0
    assert "injected" in ia.last_error()
    lib.indialign_inject_failure(0)


def test_null_pointer_rejected():
    lib = ia.load()
    arr = (abi.NativePairInput * 1)()
    arr[0].length = 10  # pointers left NULL
    res = (abi.NativePairResult * 1)()
    cfg = ia.default_config()
    assert lib.indialign_tmscore_search_batch(1, arr, ctypes.byref(cfg), res) == -4


def test_no_device_fails_loudly():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    assert ia.load().indialign_cuda_available() == 0
    with pytest.raises(ia.IndialignError, match="rc=-2"):
        ia.search(W.single(0))


def test_padded_entry_rejects_bad_lengths_before_device_work():
    lib = ia.load()
    cfg = ia.default_config()
    lens = (ctypes.c_int * 2)(10, 40)
    ln = (ctypes.c_double * 2)(10.0, 40.0)
    dummy = ctypes.c_void_p(16)  # never dereferenced: validation fails first
    rc = lib.indialign_tmscore_search_padded(2, 32, lens, dummy, dummy, dummy, dummy, dummy, ln,
                                             ctypes.byref(cfg), None, dummy)
    assert rc == -4 and "length" in ia.last_error()
    rc = lib.indialign_tmscore_search_padded(2, 0, lens, dummy, dummy, dummy, dummy, dummy, ln,
                                             ctypes.byref(cfg), None, dummy)
    assert rc == -4


def test_gemm_rejects_bad_arguments_before_device_work():
    """indialign_gemm_bf16 checks shapes, strides and alignment on the host
    before its first CUDA call: each case returns INDIALIGN_E_INPUT."""
    lib = ia.load()
    p = 1 << 12  # 16-byte aligned, never dereferenced
    cases = [
        # lda, a_mn, ldb, b_mn, m, n, k, ldc, c_trans, a_ptr
        (64, 0, 64, 0, 128, 300, 64, 300, 0, p),        # n > 256
        (60, 0, 64, 0, 128, 64, 64, 64, 0, p),          # lda not a multiple of 8
        (64, 1, 64, 0, 200, 64, 64, 64, 0, p),          # MN-major A beyond one 128-row tile
        (32, 0, 64, 0, 128, 64, 64, 64, 0, p),          # K-major lda < k
        (64, 0, 64, 0, 128, 64, 64, 64, 0, p + 2),      # operand not 16-byte aligned
        (64, 0, 64, 0, 128, 64, 64, 63, 0, p),          # ldc < n: output rows overlap
        (64, 0, 64, 0, 128, 64, 64, 127, 1, p),         # transposed store, ldc < m
        (64, 0, 64, 0, 1 << 24, 256, 64, 256, 0, p),    # m x n beyond int range
    ]
    for lda, a_mn, ldb, b_mn, m, n, k, ldc, c_trans, a in cases:
        rc = lib.indialign_gemm_bf16(a, lda, a_mn, p, ldb, b_mn, m, n, k, p, ldc, c_trans, None, 1, None)
        assert rc == -4, (lda, a_mn, m, n, k, ldc, c_trans, rc)
        assert "gemm_bf16" in ia.last_error()


def test_batch_options_layout_matches_header(tmp_path):
    """The Python mirror of IndialignBatchOptions has the C struct's size and
    field offsets (a C program compiled against the header prints them)."""
    fields = [f[0] for f in ia.BatchOptions._fields_]
    src = tmp_path / "layout.c"
    body = "\n".join(f'    printf("%s %zu\\n", "{f}", offsetof(IndialignBatchOptions, {f}));' for f in fields)
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "indialign_b200.h"\n'
                   'int main(void) {\n' + body +
                   '\n    printf("sizeof %zu\\n", sizeof(IndialignBatchOptions));\n    return 0;\n}\n')
    exe = tmp_path / "layout"
    import subprocess
    subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], check=True, capture_output=True,
                                                        text=True).stdout.splitlines())
    for f in fields:
        assert int(out[f]) == getattr(ia.BatchOptions, f).offset, f
    assert int(out["sizeof"]) == ctypes.sizeof(ia.BatchOptions)


def test_search_tensors_rejects_bad_shapes_before_device_work():
    torch = pytest.importorskip("torch")
    with pytest.raises(ValueError):
        ia.search_tensors(torch.zeros(2, 5, 3), torch.zeros(2, 6, 3))
    with pytest.raises(ValueError):
        ia.search_tensors(torch.zeros(2, 5, 3), torch.zeros(2, 5, 3))  # host tensors
