"""C1' traces from PDB text and padded pairs of unequal length; the oracle
(C restatement) against the reference build on such pairs.  (The final score
stays the reference's same-index TM-score over residues valid on both
sides, so it is not a measure of the offset correspondence.)"""
from __future__ import annotations

import numpy as np
import pytest

from indialign_b200 import abi, pdb, workloads as W


def _trace(L, seed):
    return W.make_trace(L, np.random.default_rng(seed))


def test_c1_roundtrip_and_models():
    x = _trace(30, 1)
    keep = np.ones(30, bool)
    keep[[3, 4, 17]] = False
    txt = pdb.c1_pdb_text(x, keep, chain="B", first_resnum=10)
    ch = pdb.c1_by_chain(txt)
    assert list(ch) == ["B"]
    assert sorted(ch["B"]) == [10 + i for i in range(30) if keep[i]]
    got = np.array([ch["B"][10 + i] for i in range(30) if keep[i]])
    np.testing.assert_allclose(got, x[keep], atol=5e-4)
    two = "MODEL        1\n" + txt.replace("END\n", "") + "ENDMDL\nMODEL        2\n" + \
        pdb.c1_pdb_text(x[:12]).replace("END\n", "") + "ENDMDL\nEND\n"
    models = pdb.c1_models(two)
    assert [m.shape for m in models] == [(27, 3), (12, 3)]
    assert [m.shape for m in pdb.c1_models(txt)] == [(27, 3)]


def test_extraction_rules_follow_the_reference_benchmark():
    """Records other than ATOM, other atom names and models after the first
    are ignored where the reference's extraction ignores them; atoms after
    the last ENDMDL of a multi-model file are dropped."""
    x = _trace(6, 3)
    a = pdb.c1_pdb_text(x, chain="A").replace("END\n", "")
    b = pdb.c1_pdb_text(x[:4] + 1.0, chain="B", first_resnum=20).replace("END\n", "")
    het = "HETATM    1  C1'   A A  99       1.000   2.000   3.000  1.00  0.00           C\n"
    other = a.splitlines()[0].replace(" C1' ", " C2' ") + "\n"
    text = "MODEL        1\n" + a + het + other + b + "ENDMDL\nMODEL        2\n" + a + "ENDMDL\n" + a
    models = pdb.c1_models(text)
    assert [m.shape for m in models] == [(10, 3), (6, 3)]  # trailing atoms dropped
    ch = pdb.c1_chains(text)
    assert sorted(ch) == ["A", "B"] and ch["A"].shape == (6, 3) and ch["B"].shape == (4, 3)
    np.testing.assert_allclose(ch["B"], x[:4] + 1.0, atol=5e-4)
    by = pdb.c1_by_chain(text)
    assert sorted(by["B"]) == [20, 21, 22, 23] and 99 not in by["A"]
    assert [m.shape for m in pdb.c1_models(a)] == [(6, 3)]  # no MODEL records: one model


def test_model_and_chain_extraction_ignore_the_residue_number_field():
    """A blank or non-numeric resSeq (hybrid-36 style) does not stop the model
    and chain extractors, which, like the reference benchmark's, never read
    the residue number."""
    x = _trace(5, 7)
    lines = pdb.c1_pdb_text(x, chain="A").splitlines()
    odd = [l[:22] + ("    " if k % 2 else "A0B1") + l[26:] if l.startswith("ATOM") else l
           for k, l in enumerate(lines)]
    text = "\n".join(odd) + "\n"
    models = pdb.c1_models(text)
    assert [m.shape for m in models] == [(5, 3)]
    np.testing.assert_allclose(models[0], x, atol=5e-4)
    assert pdb.c1_chains(text)["A"].shape == (5, 3)


def test_most_divergent_pair():
    rng = np.random.default_rng(4)
    base = _trace(20, 5)
    models = [base + rng.normal(0, 0.2, base.shape) for _ in range(6)]
    models[4] = base + 5.0  # far from every other model
    i, j, r = pdb.most_divergent_pair(models)
    assert 4 in (i, j) and r > 4.0
    # a large ensemble is scanned on model 0 and 19 evenly spread models
    many = [base + rng.normal(0, 0.1, base.shape) for _ in range(41)]
    many[8] = base + 9.0  # not among the scanned models (1, 3, 5, 7, 9, ...)
    many[40] = base + 3.0  # the last model is always scanned
    i, j, _ = pdb.most_divergent_pair(many)
    assert 40 in (i, j) and 8 not in (i, j)
    assert pdb.most_divergent_pair([base]) == (0, 1, -1.0)


def _ensemble_text(models, chain="A"):
    body = ""
    for k, m in enumerate(models):
        body += f"MODEL     {k + 1:>4d}\n" + pdb.c1_pdb_text(m, chain=chain).replace("END\n", "") + "ENDMDL\n"
    return body + "END\n"


def test_ensemble_pair_picks_the_most_divergent_models():
    base = _trace(40, 6)
    rng = np.random.default_rng(1)
    models = [base + rng.normal(0, 0.3, base.shape) for _ in range(5)]
    models[2] = base + rng.normal(0, 4.0, base.shape)
    pair, (i, j, r) = pdb.ensemble_pair(_ensemble_text(models))
    assert 2 in (i, j) and r > 3.0
    np.testing.assert_allclose(pair.pred, models[i], atol=5e-4)
    np.testing.assert_allclose(pair.native, models[j], atol=5e-4)
    assert pair.lnorm == 40.0 and pair.valid.all()
    assert pdb.ensemble_pair(_ensemble_text(models[:1])) is None           # one model
    assert pdb.ensemble_pair(_ensemble_text([base, base[:30]])) is None    # unequal lengths
    assert pdb.ensemble_pair(_ensemble_text([base[:20], base[:20]])) is None  # too short


def test_family_pairs_by_residue_number():
    base = _trace(60, 7)
    native = pdb.c1_pdb_text(base, chain="A") + pdb.c1_pdb_text(base[:10], chain="B")
    keep = np.ones(60, bool)
    keep[:5] = False
    pred1 = pdb.c1_pdb_text(base + 0.5, keep, chain="C")
    pred2 = pdb.c1_pdb_text(base[40:], chain="A", first_resnum=41)   # 20 residues: too short a chain
    pred3 = pdb.c1_pdb_text(base[:45], chain="D", first_resnum=30)   # 30..74: 31 shared with the native
    assert pdb.longest_chain(native)[0] == "A" and pdb.longest_chain(pred2) is None
    pairs = pdb.family_pairs([native, pred1, pred2, pred3], min_shared=20)
    assert len(pairs) == 2
    p1, p3 = pairs
    assert int(p1.valid.sum()) == 55 and p1.lnorm == 55.0 and len(p1.valid) == 60
    assert int(p3.valid.sum()) == 31 and len(p3.valid) == 74
    assert pdb.family_pairs([native, pred3], min_shared=40) == []


def test_pair_by_resnum_marks_each_side():
    a = {1: np.zeros(3), 2: np.ones(3), 5: np.full(3, 2.0)}
    b = {2: np.ones(3), 3: np.zeros(3), 5: np.zeros(3)}
    p = pdb.pair_by_resnum(a, b)
    assert p.pred.shape == (4, 3)
    assert p.pred_valid.tolist() == [1, 1, 0, 1]
    assert p.native_valid.tolist() == [0, 1, 1, 1]
    assert p.valid.tolist() == [0, 1, 0, 1] and p.lnorm == 2.0


def _cross_pairs():
    out = []
    for k, (Lp, Ln) in enumerate([(60, 48), (45, 70), (90, 90)]):
        x = _trace(max(Lp, Ln), 10 + k)
        rng = np.random.default_rng(20 + k)
        nat = x[:Ln] + rng.normal(0, 1.5, (Ln, 3))
        nat = nat @ W.random_rotation(rng).T + rng.uniform(-30, 30, 3)
        pred = x[max(Lp, Ln) - Lp:] if Lp < Ln else x[:Lp]  # a shifted segment when shorter
        out.append(pdb.pair_padded(pred, nat))
    return out


def test_cross_length_pairs_oracle_matches_reference(oracle, ref):
    pairs = _cross_pairs()
    rc, so, _, _ = abi.run_batch(oracle, pairs, prefix="ora_")
    rc2, sr, _, _ = abi.run_batch(ref, pairs)
    assert rc == 0 and rc2 == 0
    np.testing.assert_allclose(so, sr, atol=1e-9)


@pytest.mark.gpu
def test_cross_length_pairs_gpu_vs_oracle(oracle):
    import indialign_b200 as ia
    pairs = _cross_pairs()
    s, _, _ = ia.search(pairs)
    rc, so, _, _ = abi.run_batch(oracle, pairs, prefix="ora_")
    assert rc == 0
    assert np.all(s >= so - 1e-6), (s, so)
