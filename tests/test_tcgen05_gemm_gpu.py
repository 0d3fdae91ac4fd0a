"""The tcgen05 BF16 GEMM of the ranker's training backward
(indialign_gemm_bf16, k_tcgen05.cu) against an FP64 product of the same
BF16 values, through the C ABI.

Covers both operand layouts the tensor cores read from shared memory
(K-major and MN-major, each side), ragged M, N and K (the tensor maps'
zero fill), split-K with its fixed-order sum, transposed output, the three
shapes the backward uses, and the argument checks.

Tolerance: FP32 accumulation of BF16 products; |C - C64| <= 1e-5 *
sum_k |a_ik b_jk| + 1e-6 per element.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

import indialign_b200 as ia

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _bf16(torch, a):
    """Device BF16 copy of a float array and the float64 values it holds."""
    t = torch.tensor(a, dtype=torch.float32, device="cuda").to(torch.bfloat16).contiguous()
    return t, t.float().cpu().numpy().astype(np.float64)


def _gemm(torch, A, lda, a_mn, B, ldb, b_mn, m, n, k, ldc, c_trans, splits):
    lib = ia.load()
    rows, cols = (n, ldc) if c_trans else (m, ldc)
    C = torch.full((rows, cols), float("nan"), device="cuda")
    part = torch.empty(max(splits, 1) * m * n, device="cuda") if splits > 1 else None
    rc = lib.indialign_gemm_bf16(A.data_ptr(), lda, a_mn, B.data_ptr(), ldb, b_mn, m, n, k, C.data_ptr(), ldc,
                                 c_trans, part.data_ptr() if part is not None else None, splits, None)
    torch.cuda.synchronize()
    return rc, C.cpu().numpy().astype(np.float64)


CASES = [
    # a_mn, b_mn, m, n, k, splits, c_trans
    (1, 1, 128, 128, 8192, 32, 0),   # dW2 = h1^T dz2
    (0, 0, 8192, 128, 128, 1, 0),    # dh1 = dz2 W2^T
    (1, 1, 128, 16, 8192, 32, 1),    # dW1^T = dz1^T xn, stored transposed
    (0, 0, 300, 48, 200, 1, 0),
    (0, 0, 129, 256, 64, 1, 1),
    (1, 1, 100, 200, 1000, 3, 0),
    (0, 1, 257, 64, 77, 2, 0),
    (1, 0, 128, 32, 130, 1, 1),
    (1, 1, 128, 128, 77, 1, 0),
    (0, 0, 1, 16, 1, 1, 0),
]


@pytest.mark.parametrize("a_mn,b_mn,m,n,k,splits,c_trans", CASES)
def test_gemm_matches_fp64(torch_cuda, a_mn, b_mn, m, n, k, splits, c_trans):
    torch = torch_cuda
    rng = np.random.default_rng(m * 7 + n * 3 + k)
    a = rng.normal(0, 1, (m, k)).astype(np.float32)
    b = rng.normal(0, 1, (n, k)).astype(np.float32)
    # operands in the layout under test, leading dimension padded to 8
    lda = ((m if a_mn else k) + 7) // 8 * 8
    ldb = ((n if b_mn else k) + 7) // 8 * 8
    a_st = np.zeros((k, lda) if a_mn else (m, lda), np.float32)
    b_st = np.zeros((k, ldb) if b_mn else (n, ldb), np.float32)
    if a_mn:
        a_st[:, :m] = a.T
    else:
        a_st[:, :k] = a
    if b_mn:
        b_st[:, :n] = b.T
    else:
        b_st[:, :k] = b
    A, a_st64 = _bf16(torch, a_st)
    B, b_st64 = _bf16(torch, b_st)
    a64 = a_st64[:, :m].T if a_mn else a_st64[:, :k]
    b64 = b_st64[:, :n].T if b_mn else b_st64[:, :k]
    ref = a64 @ b64.T
    bound = 1e-5 * (np.abs(a64) @ np.abs(b64).T) + 1e-6
    ldc = (m if c_trans else n) + 3
    rc, C = _gemm(torch, A, lda, a_mn, B, ldb, b_mn, m, n, k, ldc, c_trans, splits)
    assert rc == 0, ia.last_error()
    got = C[:n, :m].T if c_trans else C[:m, :n]
    assert np.all(np.isfinite(got))
    err = np.abs(got - ref)
    assert np.all(err <= bound), (float(err.max()), float((err - bound).max()))
    # the padding columns of C are untouched
    assert np.all(np.isnan(C[:, (m if c_trans else n):]))


def test_gemm_rejects_what_it_does_not_take(torch_cuda):
    torch = torch_cuda
    lib = ia.load()
    A = torch.zeros(256 * 256, dtype=torch.bfloat16, device="cuda")
    C = torch.zeros(256 * 256, device="cuda")
    E = -4  # INDIALIGN_E_INPUT
    bad = [
        (64, 0, 128, 300, 64),   # n > 256
        (64, 1, 200, 64, 64),    # MN-major A with m > 128
        (60, 0, 128, 64, 64),    # lda not a multiple of 8
        (32, 0, 128, 64, 64),    # K-major lda < k
    ]
    for lda, a_mn, m, n, k in bad:
        rc = lib.indialign_gemm_bf16(A.data_ptr(), lda, a_mn, A.data_ptr(), 64, 0, m, n, k, C.data_ptr(), n, 0,
                                     None, 1, None)
        assert rc == E, (lda, a_mn, m, n, k, rc)
    # misaligned operand pointer
    rc = lib.indialign_gemm_bf16(A.data_ptr() + 2, 64, 0, A.data_ptr(), 64, 0, 128, 64, 64, C.data_ptr(), 64, 0,
                                 None, 1, None)
    assert rc == E
    # split-K without a partial buffer
    rc = lib.indialign_gemm_bf16(A.data_ptr(), 256, 0, A.data_ptr(), 256, 0, 128, 64, 256, C.data_ptr(), 64, 0,
                                 None, 4, None)
    assert rc == E
