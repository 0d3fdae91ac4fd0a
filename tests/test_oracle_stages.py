"""Stage-level pins of the oracle against the reference's own functions.

Each oracle stage function (oracle/indialign_oracle.c) is called beside the
reference function it restates, through the thin extern "C" wrappers of
oracle/ref_stages.cpp compiled from the reference's headers
(indialign_c/*.h).  Inputs are seeded synthetic pairs: a near-native pair, a
noisy pair with invalid residues, a hard pair (shared stems only) and a short
pair.  Masks, labels and alignments must be identical; scores agree to 1e-12
and rotations / translations to 1e-9.  (Measured: scores within 1e-15 and
transforms within 1e-13; about half of the stages are bit-equal, the rest
differ in the last bits because the C oracle and the C++ reference are
compiled with different floating-point contraction.)

CPU only; skipped when the reference build (oracle/_ref) is absent.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from indialign_b200 import workloads

TOL = 1e-12


def _arg(a):
    if isinstance(a, np.ndarray):
        assert a.flags.c_contiguous
        return ctypes.c_void_p(a.ctypes.data)
    if isinstance(a, float):
        return ctypes.c_double(a)
    if isinstance(a, (bool, int, np.integer)):
        return ctypes.c_int(int(a))
    if isinstance(a, ctypes.Array):
        return a
    raise TypeError(type(a))


def call(fn, *args, restype=None):
    fn.restype = restype
    return fn(*[_arg(a) for a in args])


def _pairs():
    rng = np.random.default_rng(20240611)
    return {
        "near": workloads.make_pair(72, 1.0, rng),
        "noisy_masked": workloads.make_pair(110, 6.0, rng, invalid_frac=0.08),
        "hard": workloads.make_pair(140, 1.5, rng, invalid_frac=0.03, hard=True),
        "short": workloads.make_pair(12, 3.0, rng),
    }


PAIRS = _pairs()


@pytest.fixture(scope="module")
def ora(oracle):
    """A private handle on the oracle library: other modules set argtypes on
    the shared one, this module passes untyped pointers."""
    return ctypes.CDLL(oracle._name)


@pytest.fixture(scope="module")
def ref(ref_stages):
    return ctypes.CDLL(ref_stages._name)


@pytest.fixture(params=sorted(PAIRS))
def pair(request):
    return PAIRS[request.param]


def _d0(lib, prefix, L):
    d0, d0s, sd8 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    getattr(lib, prefix + "d0")(ctypes.c_double(L), ctypes.byref(d0), ctypes.byref(d0s), ctypes.byref(sd8))
    return d0.value, d0s.value, sd8.value


def _flat(pr):
    p = np.ascontiguousarray(pr.pred, np.float64).reshape(-1)
    q = np.ascontiguousarray(pr.native, np.float64).reshape(-1)
    return p, q, pr.valid.copy(), pr.pred_valid.copy(), pr.native_valid.copy(), len(pr.valid)


def _same13(a, b):
    assert a[0] == pytest.approx(b[0], abs=TOL), (a[0], b[0])
    np.testing.assert_allclose(a[1:], b[1:], atol=1e-9, rtol=0)


def test_d0_scales(ora, ref):
    lib = ora
    for L in (1.0, 5.0, 12.0, 19.0, 21.0, 30.0, 31.0, 40.0, 64.0, 300.0, 1500.0, 8192.0):
        assert _d0(lib, "ora_", L) == _d0(ref, "ref_", L)


def test_kabsch_and_tm_score(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    rng = np.random.default_rng(N)
    for mask in (v, (rng.uniform(size=N) < 0.3).astype(np.uint8) & v):
        R1, t1, R2, t2 = (np.zeros(k) for k in (9, 3, 9, 3))
        call(lib.ora_kabsch, p, q, mask, N, R1, t1)
        call(ref.ref_kabsch, p, q, mask, N, R2, t2)
        np.testing.assert_allclose(R1, R2, atol=1e-12, rtol=0)
        np.testing.assert_allclose(t1, t2, atol=1e-10, rtol=0)
        for use_d8 in (0, 1):
            s1 = call(lib.ora_tm_score, p, q, v, R1, t1, d0, pair.lnorm, sd8, N, use_d8, restype=ctypes.c_double)
            s2 = call(ref.ref_tm_score, p, q, v, R1, t1, d0, pair.lnorm, sd8, N, use_d8,
                      restype=ctypes.c_double)
            assert s1 == pytest.approx(s2, abs=TOL)


def test_cov_to_rotation(ora, ref):
    rng = np.random.default_rng(3)
    cases = [rng.standard_normal(9) for _ in range(20)]
    cases += [np.diag([3.0, 2.0, 1.0]).reshape(-1), np.diag([1.0, 1.0, -1.0]).reshape(-1),
              np.zeros(9), np.outer([1.0, 2.0, 3.0], [0.5, -1.0, 2.0]).reshape(-1)]
    for H in cases:
        H = np.ascontiguousarray(H)
        R1, R2 = np.zeros(9), np.zeros(9)
        call(ora.ora_cov_to_rotation, H, R1)
        call(ref.ref_cov_to_rotation, H, R2)
        np.testing.assert_allclose(R1, R2, atol=1e-12, rtol=0)


@pytest.mark.parametrize("Np,Nn", [(1, 1), (7, 13), (40, 40), (57, 31)])
def test_nw_dp_and_traceback(ora, ref, Np, Nn):
    rng = np.random.default_rng(Np * 100 + Nn)
    smat = rng.uniform(0, 1, Np * Nn)
    smat[rng.uniform(size=smat.size) < 0.2] = 0.5  # ties in the max
    for gap in (-0.6, 0.0):
        H1, H2 = np.zeros((Np + 1) * (Nn + 1)), np.zeros((Np + 1) * (Nn + 1))
        T1, T2 = np.zeros(H1.size, np.int8), np.zeros(H1.size, np.int8)
        call(ora.ora_nw_dp, smat, Np, Nn, gap, H1, T1)
        call(ref.ref_nw_dp, smat, Np, Nn, gap, H2, T2)
        np.testing.assert_array_equal(T1, T2)
        np.testing.assert_allclose(H1, H2, atol=TOL, rtol=0)
        m = min(Np, Nn)
        a1, b1, a2, b2 = (np.zeros(m, np.int32) for _ in range(4))
        n1 = call(ora.ora_nw_align, smat, Np, Nn, gap, a1, b1, restype=ctypes.c_int)
        n2 = call(ref.ref_nw_align, smat, Np, Nn, gap, a2, b2, restype=ctypes.c_int)
        assert n1 == n2
        np.testing.assert_array_equal(a1[:n1], a2[:n2])
        np.testing.assert_array_equal(b1[:n1], b2[:n2])


def test_seed_masks(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    cap = 4096
    for use_frag in (0, 1):
        for max_starts in (1, 3, 50):  # max_starts 0 divides by zero in both
            m1, m2 = np.zeros(cap * N, np.uint8), np.zeros(cap * N, np.uint8)
            k1 = call(lib.ora_seed_masks, N, v, use_frag, max_starts, m1, cap, restype=ctypes.c_int)
            k2 = call(ref.ref_seed_masks, N, v, use_frag, max_starts, m2, cap, restype=ctypes.c_int)
            assert k1 == k2 and k1 > 0
            np.testing.assert_array_equal(m1[:k1 * N], m2[:k2 * N])
        m1, m2 = np.zeros(cap * N, np.uint8), np.zeros(cap * N, np.uint8)
        k1 = call(lib.ora_all_seeds, p, q, v, N, d0s, d0, use_frag, m1, cap, restype=ctypes.c_int)
        k2 = call(ref.ref_all_seeds, p, q, v, N, d0s, d0, use_frag, m2, cap, restype=ctypes.c_int)
        assert k1 == k2 and k1 > 0
        np.testing.assert_array_equal(m1[:k1 * N], m2[:k2 * N])


def _seeds(lib, pair):
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    cap = 4096
    m = np.zeros(cap * N, np.uint8)
    K = call(lib.ora_all_seeds, p, q, v, N, d0s, d0, 1, m, cap, restype=ctypes.c_int)
    return m[:K * N].copy(), K


def test_seed_refine(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    seeds, K = _seeds(lib, pair)
    for k in sorted({0, K // 3, K // 2, K - 1}):
        seed = np.ascontiguousarray(seeds[k * N:(k + 1) * N])
        for max_iter in (1, 20):
            R1, t1, R2, t2 = (np.zeros(k_) for k_ in (9, 3, 9, 3))
            call(lib.ora_seed_refine, p, q, v, seed, d0s, N, max_iter, R1, t1)
            call(ref.ref_iterative_seed_refine, p, q, v, seed, d0s, N, max_iter, R2, t2)
            np.testing.assert_allclose(R1, R2, atol=1e-12, rtol=0)
            np.testing.assert_allclose(t1, t2, atol=1e-10, rtol=0)


def test_seed_bank(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    seeds, K = _seeds(lib, pair)
    cands = np.zeros(16)
    C = call(lib.ora_d0_candidates, d0, d0s, cands, restype=ctypes.c_int)
    for use_d8, early in ((1, 1.1), (0, 1.1), (1, 0.5)):
        o1, o2 = np.zeros(13), np.zeros(13)
        call(lib.ora_seed_bank, p, q, v, seeds, K, cands, C, d0, sd8, pair.lnorm, N, 20, use_d8, early, o1)
        call(ref.ref_seed_bank, p, q, v, seeds, K, cands, C, d0, sd8, pair.lnorm, N, 20, use_d8,
             early, o2)
        _same13(o1, o2)


def test_assign_ss(ora, ref, pair):
    p, q, v, pv, nv, N = _flat(pair)
    for xyz, m in ((p, pv), (q, nv)):
        s1 = ctypes.create_string_buffer(N + 1)
        s2 = ctypes.create_string_buffer(N + 1)
        call(ora.ora_assign_ss, xyz, m, N, s1)
        call(ref.ref_assign_ss, xyz, m, N, s2)
        assert s1.raw[:N] == s2.raw[:N]


def test_rescue_stages(ora, ref, pair):
    """Gapless threading, local fragment DP (normal and dense), threading DP."""
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    L = pair.lnorm
    o1, o2 = np.zeros(13), np.zeros(13)
    call(lib.ora_gapless, p, q, pv, nv, v, d0, d0s, L, N, o1)
    call(ref.ref_gapless, p, q, pv, nv, v, d0, d0s, L, N, o2)
    _same13(o1, o2)
    for dense in (0, 1):
        o1, o2 = np.zeros(13), np.zeros(13)
        call(lib.ora_local_fragment_dp, p, q, pv, nv, d0, d0s, L, N, dense, o1)
        call(ref.ref_local_fragment_dp, p, q, v, pv, nv, d0, d0s, L, N, dense, o2)
        _same13(o1, o2)
    o1, o2 = np.zeros(13), np.zeros(13)
    call(lib.ora_threading_dp, p, q, pv, nv, d0, d0s, L, N, o1)
    call(ref.ref_threading_dp, p, q, v, pv, nv, d0, d0s, L, N, o2)
    _same13(o1, o2)


def _start(lib, pair):
    """A mediocre superposition to refine from: Kabsch on every third residue
    of a perturbed copy."""
    p, q, v, pv, nv, N = _flat(pair)
    rng = np.random.default_rng(N + 1)
    qq = (q.reshape(-1, 3) + rng.standard_normal((N, 3)) * 4.0).reshape(-1).copy()
    mask = np.zeros(N, np.uint8)
    mask[::3] = 1
    mask &= v
    R, t = np.zeros(9), np.zeros(3)
    call(lib.ora_kabsch, p, qq, mask, N, R, t)
    return R, t


def test_dp_refine(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    R0, t0 = _start(lib, pair)
    for max_iter, lite in ((3, 0), (3, 1), (1, 0)):
        o1, o2 = np.zeros(13), np.zeros(13)
        call(lib.ora_dp_refine, p, q, pv, nv, R0, t0, d0, d0s, sd8, pair.lnorm, N, max_iter, lite, o1)
        call(ref.ref_dp_refine, p, q, v, pv, nv, R0, t0, d0, d0s, sd8, pair.lnorm, N, max_iter, lite,
             o2)
        _same13(o1, o2)


def test_detailed_search(ora, ref, pair):
    """Detailed search over an NW alignment of the start superposition, and
    over the identity correspondence."""
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    ident = np.flatnonzero(v).astype(np.int32)
    rng = np.random.default_rng(N + 2)
    sub = np.sort(rng.choice(ident, size=max(1, ident.size * 2 // 3), replace=False)).astype(np.int32)
    shifted = sub[sub + 2 < N]
    for ap, an in ((ident, ident.copy()), (sub, sub.copy()), (shifted, (shifted + 2).astype(np.int32))):
        ap, an = np.ascontiguousarray(ap), np.ascontiguousarray(an)
        na = int(ap.size)
        for use_frag, mio, ms in ((1, -1, 50), (0, -1, 50), (1, 2, 3)):
            o1, o2 = np.zeros(13), np.zeros(13)
            call(lib.ora_detailed_search, p, q, ap, an, na, d0, d0s, sd8, pair.lnorm, use_frag, mio, ms, o1)
            call(ref.ref_detailed_search, p, q, ap, an, na, d0, d0s, sd8, pair.lnorm, N, use_frag, mio,
                 ms, o2)
            _same13(o1, o2)


def test_topk_seed(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    R, t = _start(lib, pair)
    P = p.reshape(-1, 3) @ R.reshape(3, 3).T + t
    d2 = np.ascontiguousarray(((P - q.reshape(-1, 3)) ** 2).sum(1))
    d2[:: 5] = d2[0]  # ties
    for frac in (0.5, 0.25, 1.0):
        m1, m2 = np.zeros(N, np.uint8), np.zeros(N, np.uint8)
        call(lib.ora_topk_seed, d2, v, N, frac, m1)
        call(ref.ref_topk_seed, d2, v, N, frac, m2)
        np.testing.assert_array_equal(m1, m2)


def test_weighted_refine(ora, ref, pair):
    lib = ora
    p, q, v, pv, nv, N = _flat(pair)
    d0, d0s, sd8 = _d0(lib, "ora_", pair.lnorm)
    R0, t0 = _start(lib, pair)
    for iters in (1, 5):
        R1, t1, R2, t2 = R0.copy(), t0.copy(), R0.copy(), t0.copy()
        s1, s2 = ctypes.c_double(-1.0), ctypes.c_double(-1.0)
        lib.ora_weighted_refine.restype = None
        lib.ora_weighted_refine(*[_arg(a) for a in (p, q, v, d0, pair.lnorm, N, iters, R1, t1)], ctypes.byref(s1))
        ref.ref_weighted_refine.restype = None
        ref.ref_weighted_refine(*[_arg(a) for a in (p, q, v, d0, pair.lnorm, N, iters, R2, t2)],
                                       ctypes.byref(s2))
        assert s1.value == pytest.approx(s2.value, abs=TOL)
        np.testing.assert_allclose(R1, R2, atol=1e-9, rtol=0)
        np.testing.assert_allclose(t1, t2, atol=1e-9, rtol=0)


# ---- candidate schedules of the learned ranker's oracle ---------------------

def _ranker_oracle():
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import ranker_oracle
    return ranker_oracle


def _ref_list(fn, *args, cap=4096):
    out = np.zeros(cap, np.int32)
    fn.restype = ctypes.c_int
    k = fn(*[ctypes.c_int(a) for a in args], ctypes.c_void_p(out.ctypes.data), ctypes.c_int(cap))
    assert k >= 0
    return out[:k].tolist()


SIZES = list(range(0, 80)) + [99, 100, 101, 149, 150, 151, 199, 200, 201, 249, 250, 251, 299, 300, 301,
                              349, 350, 351, 512, 999, 1000, 1500, 8192]


def test_ranker_schedules_match_reference(ref):
    """local_frag_lengths / local_jump (rescue.h:12-46), fragment_lengths and
    start_positions (seeds.h:15-37) as the ranker oracle restates them."""
    ro = _ranker_oracle()
    for L in SIZES:
        for dense in (0, 1):
            ref.ref_local_jump.restype = ctypes.c_int
            assert ro.local_jump(L, bool(dense)) == ref.ref_local_jump(ctypes.c_int(L), ctypes.c_int(dense)), L
        assert ro.frag_lengths(L) == _ref_list(ref.ref_fragment_lengths, L), L
        for frag in sorted({1, 4, 8, max(1, L // 2), max(1, L)}):
            for ms in (1, 5, 50):
                assert ro.start_positions(L, frag, ms) == _ref_list(ref.ref_start_positions, L, frag, ms), \
                    (L, frag, ms)
    for plen in (3, 4, 12, 13, 40, 77, 150, 300, 1000):
        for nlen in (3, 4, 12, 13, 40, 77, 150, 300, 1000):
            for dense in (0, 1):
                assert ro.local_frag_lengths(plen, nlen, bool(dense)) == \
                    _ref_list(ref.ref_local_frag_lengths, plen, nlen, dense), (plen, nlen, dense)


@pytest.mark.parametrize("na", [3, 4, 7, 16, 33, 64, 100, 257])
def test_ranker_detailed_seeds_match_reference_masks(ref, na):
    """The ranker oracle's detailed-search seeds (whole aligned set, then the
    fragment windows) are the masks the reference's build_seed_masks makes on
    an all-valid aligned set of na points (align.h:33-37)."""
    ro = _ranker_oracle()
    cap = 8192
    masks = np.zeros(cap * na, np.uint8)
    ones = np.ones(na, np.uint8)
    K = call(ref.ref_seed_masks, na, ones, 1, 50, masks, cap, restype=ctypes.c_int)
    masks = masks[:K * na].reshape(K, na)
    want = []
    for row in masks:
        idx = np.flatnonzero(row)
        assert idx.size and idx[-1] - idx[0] + 1 == idx.size  # one contiguous window
        want.append((int(idx.size), int(idx[0]), int(idx[0])))
    assert ro.det_seeds(na) == want
