"""The oracle (oracle/indialign_oracle.c) pinned against the reference.

The golden fixtures hold the reference build's own outputs (see
tests/golden/make_golden.py); when the reference build itself is present
(oracle/_ref) the oracle is also compared with it on fresh inputs."""
import ctypes

import numpy as np
import pytest

from conftest import GoldenPairs, rot_err_deg
from indialign_b200 import abi, workloads as W


def test_oracle_matches_golden(oracle, golden):
    rc, s, R, t = abi.run_batch(oracle, golden.pairs, prefix="ora_")
    assert rc == 0
    # same FP64 algorithm; only reassociation under -ffast-math differs
    np.testing.assert_allclose(s, golden.score, rtol=0, atol=1e-9)
    assert rot_err_deg(R, golden.R).max() < 1e-4


def test_oracle_stage_trace_matches_golden(oracle, golden):
    lib = oracle
    lib.ora_trace_search.argtypes = [ctypes.POINTER(abi.NativePairInput),
                                     ctypes.POINTER(abi.NativeConfig),
                                     ctypes.POINTER(ctypes.c_double),
                                     ctypes.POINTER(abi.NativePairResult)]
    cfg = abi.default_config(lib, "ora_")
    pk = abi.PackedInputs(golden.pairs)
    for k in range(pk.n):
        buf = np.zeros(10 * 13)
        res = abi.NativePairResult()
        lib.ora_trace_search(ctypes.byref(pk.arr[k]), ctypes.byref(cfg),
                             buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                             ctypes.byref(res))
        tr = buf.reshape(10, 13)
        ref = golden.trace[k]
        ran = ref[:, 0] > -1e30
        assert np.array_equal(tr[:, 0] > -1e30, ran)
        np.testing.assert_allclose(tr[ran, 0], ref[ran, 0], rtol=0, atol=1e-9)


@pytest.mark.parametrize("name,k", [("cfg1", 10), ("cfg2", 4)])
def test_oracle_matches_golden_workload_shapes(oracle, name, k):
    """The oracle on the shortest pairs of the workload-shape samples (the
    long ones are checked on the GPU against the same fixtures)."""
    g = GoldenPairs(name)
    idx = g.shortest(k)
    rc, s, R, t = abi.run_batch(oracle, [g.pairs[i] for i in idx], prefix="ora_")
    assert rc == 0
    np.testing.assert_allclose(s, g.score[idx], rtol=0, atol=1e-9)


def test_cfg2_sample_reaches_the_dense_rescue():
    """The hard pairs of the uneven sample fall below 0.3 before the dense
    local-fragment pass (so it runs) at every rescue stride bracket."""
    g = GoldenPairs("cfg2")
    # trace stage 5 = dense_local_fragment: recorded only when the pass ran
    gated = [g.pairs[k].pred.shape[0] for k in range(len(g.pairs)) if g.hard[k] and g.trace[k, 5, 0] > -1e30]
    assert len(gated) >= 6 and max(gated) >= 1000, gated


def test_sort_tie_order_matches_std_sort(oracle):
    """The anchor candidates' tie order (count-only std::sort) is reproduced."""
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_sort.npz"))
    oracle.ora_introsort_desc.argtypes = [ctypes.POINTER(ctypes.c_int)] * 2 + [ctypes.c_int]
    j = 0
    while f"keys{j}" in z:
        keys = z[f"keys{j}"].astype(np.int32).copy()
        idx = np.arange(len(keys), dtype=np.int32)
        oracle.ora_introsort_desc(keys.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                  idx.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), len(keys))
        np.testing.assert_array_equal(idx, z[f"order{j}"])
        j += 1
    assert j >= 5


def test_oracle_vs_reference_fresh(oracle, ref):
    pairs = W.batch(6, 40, 90, seed=909) + W.hard(4, seed=910)[:2]
    pairs = [p for p in pairs if p.pred.shape[0] <= 100]
    rc1, s1, R1, _ = abi.run_batch(ref, pairs)
    rc2, s2, R2, _ = abi.run_batch(oracle, pairs, prefix="ora_")
    assert rc1 == rc2 == 0
    np.testing.assert_allclose(s2, s1, rtol=0, atol=1e-9)


def test_oracle_length_zero(oracle):
    inp = abi.NativePairInput()
    inp.length = 0
    cfg = abi.default_config(oracle, "ora_")
    out = abi.NativePairResult()
    out.score = 7.0
    assert oracle.ora_tmscore_search(ctypes.byref(inp), ctypes.byref(cfg), ctypes.byref(out)) == -1
    assert out.score == 7.0


def test_oracle_non_finite_coordinates_vs_reference(oracle, ref):
    """NaN and Inf coordinates: the same final scores as the reference build.
    A NaN reaches every candidate score, nothing beats the initial -1e30, and
    the reference then returns an uninitialised (R, t) (indialign_c/search.h:
    69-70 sets only best.score), so (R, t) are compared only where a
    candidate was accepted."""
    rng = np.random.default_rng(3)
    pairs = []
    for k in range(5):
        p = W.make_pair(50, 2.0, rng)
        if k == 0:
            p.pred[7, 1] = np.nan
        elif k == 1:
            p.native[20, 0] = np.nan
        elif k == 2:
            p.pred[:, :] = np.nan
        elif k == 3:
            p.native[5, 2] = np.inf
        else:
            p.pred[3, 0] = -np.inf
        pairs.append(p)
    rc, so, Ro, to = abi.run_batch(oracle, pairs, prefix="ora_")
    rc2, sr, Rr, tr = abi.run_batch(ref, pairs)
    assert rc == 0 and rc2 == 0
    np.testing.assert_allclose(so, sr, atol=1e-12, rtol=0)
    assert np.all(so[:3] == -1e30) and np.all(sr[:3] == -1e30)
    ok = so > -1e29
    np.testing.assert_allclose(Ro[ok], Rr[ok], atol=1e-9)
    np.testing.assert_allclose(to[ok], tr[ok], atol=1e-7)


def _nw_cases():
    import os
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_nw.npz"))
    k = 0
    while f"q{k}" in z:
        yield z[f"q{k}"].astype(np.float64) / 4096.0, float(z[f"g{k}"][0]), z[f"ap{k}"], z[f"an{k}"]
        k += 1


def test_oracle_nw_matches_golden(oracle):
    oracle.ora_nw_align.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.c_int,
                                    ctypes.c_double, ctypes.POINTER(ctypes.c_int),
                                    ctypes.POINTER(ctypes.c_int)]
    n = 0
    for m, gap, ap, an in _nw_cases():
        m = np.ascontiguousarray(m)
        a = np.zeros(min(m.shape), np.int32)
        b = np.zeros(min(m.shape), np.int32)
        na = oracle.ora_nw_align(m.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), m.shape[0], m.shape[1],
                                 gap, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                 b.ctypes.data_as(ctypes.POINTER(ctypes.c_int)))
        np.testing.assert_array_equal(a[:na], ap)
        np.testing.assert_array_equal(b[:na], an)
        n += 1
    assert n >= 90
