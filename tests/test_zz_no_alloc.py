"""The allocation-free NW entry point against the allocating one.

indialign_nw_align_noalloc serves callers that may not allocate device memory
when they align (a framework's pool allocator owns all device memory, or the
path forbids driver allocations): its scratch is a fixed device array instead
of a cudaMalloc.  This file is collected last on purpose, so a failure
here never hides the rest of the suite.
"""
import ctypes
import os

import numpy as np
import pytest

import indialign_b200 as ia

pytestmark = pytest.mark.gpu
SIG = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_void_p,
       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


def _cases():
    """Golden NW cases of at least 8000 cells: (matrix, gap, reference
    alignment (ap, an)) from the reference's nw_dp + nw_traceback."""
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_nw.npz"))
    picks = []
    k = 0
    while f"q{k}" in z:
        q = z[f"q{k}"]
        if q.shape[0] * q.shape[1] >= 8000:
            picks.append((q.astype(np.float64) / 4096.0, float(z[f"g{k}"][0]), z[f"ap{k}"], z[f"an{k}"]))
        k += 1
    return picks


def _run(fn, torch, m, gap):
    d = torch.from_numpy(np.ascontiguousarray(m)).cuda()
    npr, nn = m.shape
    ap = torch.full((min(npr, nn),), -7, dtype=torch.int32, device="cuda")
    an = torch.full_like(ap, -7)
    na = torch.zeros(1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = fn(d.data_ptr(), npr, nn, gap, ap.data_ptr(), an.data_ptr(), na.data_ptr(), None)
    n = int(na.item())
    return rc, ap[:n].cpu().numpy(), an[:n].cpu().numpy()


def test_noalloc_matches_allocating_entry_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    lib = ia.load()
    for name in ("indialign_nw_align", "indialign_nw_align_noalloc"):
        getattr(lib, name).argtypes = SIG
        getattr(lib, name).restype = ctypes.c_int
    cases = _cases()
    assert len(cases) >= 2
    # calls in a row through the shared scratch, different shapes; each result
    # equals the allocating entry's and the reference's own alignment
    for m, gap, ap_ref, an_ref in (cases[-1], cases[0], cases[len(cases) // 2]):
        rc_a, ap_a, an_a = _run(lib.indialign_nw_align, torch, m, gap)
        rc_b, ap_b, an_b = _run(lib.indialign_nw_align_noalloc, torch, m, gap)
        assert rc_a == 0 and rc_b == 0
        np.testing.assert_array_equal(ap_b, ap_a)  # integer indices: exact
        np.testing.assert_array_equal(an_b, an_a)
        np.testing.assert_array_equal(ap_b, ap_ref)
        np.testing.assert_array_equal(an_b, an_ref)


def test_noalloc_at_its_size_limit():
    """A 2048 x 2048 problem (the fixed scratch's maximum) and a smaller one
    after it, both equal to the allocating entry's result."""
    torch = pytest.importorskip("torch")
    lib = ia.load()
    for name in ("indialign_nw_align", "indialign_nw_align_noalloc"):
        getattr(lib, name).argtypes = SIG
        getattr(lib, name).restype = ctypes.c_int
    rng = np.random.default_rng(11)
    for npr, nn, gap in ((2048, 2048, -0.6), (2048, 1999, 0.0), (700, 2048, -0.6)):
        q = np.where(rng.uniform(size=(npr, nn)) < 0.4, rng.integers(0, 4096, (npr, nn)), 0)
        m = q.astype(np.float64) / 4096.0
        rc_a, ap_a, an_a = _run(lib.indialign_nw_align, torch, m, gap)
        rc_b, ap_b, an_b = _run(lib.indialign_nw_align_noalloc, torch, m, gap)
        assert rc_a == 0 and rc_b == 0
        assert ap_a.size > 0
        np.testing.assert_array_equal(ap_b, ap_a)
        np.testing.assert_array_equal(an_b, an_a)


def test_noalloc_rejects_sizes_beyond_its_limit():
    torch = pytest.importorskip("torch")
    lib = ia.load()
    lib.indialign_nw_align_noalloc.argtypes = SIG
    lib.indialign_nw_align_noalloc.restype = ctypes.c_int
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.int32, device="cuda")
    for npr, nn in ((2049, 4), (4, 2049), (0, 4)):
        rc = lib.indialign_nw_align_noalloc(buf.data_ptr(), npr, nn, 0.0, out.data_ptr(),
                                            out.data_ptr(), out.data_ptr(), None)
        assert rc == -4
        assert "2048" in ia.last_error()
