"""The common-scorer comparison harness (indialign_b200/compare.py), on the
CPU: the common d0 is the reference's RNA d0, the common scorer equals the
reference's no-d8 TM-score, the USalign output parsing, the USalign call
through a stand-in executable, and a whole comparison with the oracle
standing in for the GPU search."""
from __future__ import annotations

import ctypes
import os
import stat
import sys
import textwrap

import numpy as np
import pytest

from conftest import REF_STAGES_SO, ROOT

from indialign_b200 import abi, compare as C, workloads as W

needs_ref = pytest.mark.skipif(not os.path.exists(REF_STAGES_SO), reason="reference build (oracle/_ref) not present")


@needs_ref
def test_common_d0_is_the_reference_rna_d0():
    st = ctypes.CDLL(REF_STAGES_SO)
    for L in [x * 0.5 for x in range(1, 4001)]:
        d0, d0s, sd8 = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        st.ref_d0(ctypes.c_double(L), ctypes.byref(d0), ctypes.byref(d0s), ctypes.byref(sd8))
        assert C.d0_rna(L) == d0.value, L


@needs_ref
def test_common_scorer_is_the_reference_no_d8_score():
    st = ctypes.CDLL(REF_STAGES_SO)
    st.ref_tm_score.restype = ctypes.c_double
    rng = np.random.default_rng(2)
    for p in C.fair_pairs(6, seed=3):
        R9 = W.random_rotation(rng).reshape(-1).copy()
        t = rng.normal(0, 5, 3)
        n = len(p.valid)
        d0 = C.d0_rna(p.lnorm)
        arrs = [np.ascontiguousarray(a) for a in (p.pred.reshape(-1), p.native.reshape(-1), p.valid, R9, t)]
        ref = st.ref_tm_score(*[ctypes.c_void_p(a.ctypes.data) for a in arrs], ctypes.c_double(d0),
                              ctypes.c_double(p.lnorm), ctypes.c_double(0.0), ctypes.c_int(n), ctypes.c_int(0))
        got = C.common_tm(p.pred, p.native, C.matrix_from_result(R9), t, d0, p.lnorm)
        assert got == pytest.approx(ref, abs=1e-12)


MATRIX = """\
------ The rotation matrix to rotate Structure_1 to Structure_2 ------
m               t[m]        u[m][0]        u[m][1]        u[m][2]
0       1.5000000000   0.0000000000  -1.0000000000   0.0000000000
1      -2.2500000000   1.0000000000   0.0000000000   0.0000000000
2       0.1250000000   0.0000000000   0.0000000000   1.0000000000

Code for rotating Structure 1 from (x,y,z) to (X,Y,Z):
"""


def test_usalign_output_parsing():
    M, t = C.parse_usalign_matrix(MATRIX)
    np.testing.assert_array_equal(M, [[0, -1, 0], [1, 0, 0], [0, 0, 1]])
    np.testing.assert_array_equal(t, [1.5, -2.25, 0.125])
    out = "Name of Structure_1: a\nTM-score= 0.41234 (normalized by length of Structure_1)\n" \
          "TM-score= 0.45678 (normalized by length of Structure_2)\n"
    assert C.parse_usalign_scores(out) == 0.45678
    assert C.parse_usalign_scores("no scores") == 0.0


def _fake_usalign(tmp_path):
    """A stand-in executable: checks the arguments, writes the rotation file
    and prints two scores."""
    exe = tmp_path / "fake_usalign"
    exe.write_text(textwrap.dedent(f"""\
        #!{sys.executable}
        import sys
        a = sys.argv[1:]
        assert a[2:6] == ["-atom", " C1'", "-TMscore", "1"] and a[6] == "-m", a
        assert open(a[0]).read().startswith("ATOM") and open(a[1]).read().startswith("ATOM")
        open(a[7], "w").write({MATRIX!r})
        print("TM-score= 0.25000 (normalized by length of Structure_1)")
        print("TM-score= 0.50000 (normalized by length of Structure_2)")
        """))
    exe.chmod(exe.stat().st_mode | stat.S_IXUSR)
    return str(exe)


def test_run_usalign_through_a_stand_in(tmp_path):
    p = C.fair_pairs(1, seed=5)[0]
    score, M, t, dt = C.run_usalign(p.pred, p.native, _fake_usalign(tmp_path))
    assert score == 0.5 and dt >= 0
    np.testing.assert_array_equal(t, [1.5, -2.25, 0.125])
    assert M[0, 1] == -1


@needs_ref
def test_whole_comparison_with_the_oracle_as_search(oracle, tmp_path):
    pairs = C.fair_pairs(12, seed=8)

    def search(ps):
        rc, s, R, t = abi.run_batch(oracle, ps, prefix="ora_")
        assert rc == 0
        return s, R, t

    rep = C.compare(pairs, _fake_usalign(tmp_path), search=search)
    # all residues valid and the same d0: the search's own score is the common score
    np.testing.assert_allclose(rep.self_ours, rep.common_ours, atol=1e-12)
    assert rep.stats["pairs"] == 12 and rep.stats["wins"] + rep.stats["losses"] + rep.stats["ties"] == 12
    assert rep.self_usalign.tolist() == [0.5] * 12
    assert sum(s["pairs"] for s in rep.stats["strata"]) == 12
    text = C.format_report(rep)
    assert "wins" in text and "USalign" in text
    assert "not run" in C.format_report(C.compare(pairs[:2], None, search=search))


def test_masked_common_scorer():
    rng = np.random.default_rng(9)
    p = C.fair_pairs(1, seed=4)[0]
    M, t = W.random_rotation(rng), rng.normal(0, 3, 3)
    v = (rng.uniform(size=len(p.valid)) < 0.7).astype(np.uint8)
    d0 = C.d0_rna(int(v.sum()))
    full = C.common_tm(p.pred[v != 0], p.native[v != 0], M, t, d0, float(v.sum()))
    assert C.common_tm_masked(p.pred, p.native, v, M, t, d0) == pytest.approx(full, abs=1e-14)
    assert C.common_tm_masked(p.pred, p.native, np.zeros_like(v), M, t, d0) == 0.0


@needs_ref
def test_comparison_on_padded_pdb_pairs(oracle, tmp_path):
    """Family pairs with residues missing on either side: the search's own
    score is the masked common score (same d0 of the shared count)."""
    from indialign_b200 import pdb
    rng = np.random.default_rng(12)
    x = C.random_walk_trace(70, rng)
    keep = np.ones(70, bool)
    keep[[2, 3, 40]] = False
    texts = [pdb.c1_pdb_text(x), pdb.c1_pdb_text(x @ W.random_rotation(rng).T + rng.normal(0, 2, x.shape), keep),
             pdb.c1_pdb_text(x[10:] + rng.normal(0, 3, (60, 3)), first_resnum=11)]
    pairs = pdb.family_pairs(texts)
    assert len(pairs) == 2

    def search(ps):
        rc, s, R, t = abi.run_batch(oracle, ps, prefix="ora_")
        assert rc == 0
        return s, R, t

    rep = C.compare(pairs, _fake_usalign(tmp_path), search=search)
    np.testing.assert_allclose(rep.self_ours, rep.common_ours, atol=1e-12)


def test_pdb_pairs_from_files(tmp_path):
    from indialign_b200 import pdb
    rng = np.random.default_rng(13)
    x = C.random_walk_trace(40, rng)
    ens = tmp_path / "ens.pdb"
    ens.write_text("".join(f"MODEL     {k + 1:>4d}\n" + pdb.c1_pdb_text(x + rng.normal(0, 1 + 2 * k, x.shape))
                           .replace("END\n", "") + "ENDMDL\n" for k in range(3)) + "END\n")
    fam = [tmp_path / f"f{k}.pdb" for k in range(3)]
    for k, f in enumerate(fam):
        f.write_text(pdb.c1_pdb_text(x + rng.normal(0, 1, x.shape)))
    pairs = C.pdb_pairs([str(ens)], [str(f) for f in fam])
    assert len(pairs) == 3 and all(p.valid.sum() == 40 for p in pairs)
