"""The kernel-shape table of the length buckets (host side, no device work):
the file format the library reads (tune_b200.txt / INDIALIGN_TUNE_TABLE),
its fallback to the built-in rows, and the row checks of
indialign_set_tuning."""
from __future__ import annotations

import copy

import pytest

import indialign_b200 as ia


@pytest.fixture
def restore_table(monkeypatch):
    before = ia.get_tuning()
    yield monkeypatch
    monkeypatch.delenv("INDIALIGN_TUNE_TABLE", raising=False)
    ia.set_tuning(before)


def _table(split=1, min_pairs=10):
    rows = [dict(max_len=100, bank_chunk=128, bank_cutoff_major=0, chain_chunk=8, chain_smem_trace=0),
            dict(max_len=400, bank_chunk=512, bank_cutoff_major=1, chain_chunk=32, chain_smem_trace=1),
            dict(max_len=65535, bank_chunk=256, bank_cutoff_major=1, chain_chunk=16, chain_smem_trace=1)]
    return {"split": split, "min_pairs": min_pairs, "rows": rows}


def test_table_file_round_trip(tmp_path, restore_table):
    t = _table(split=0, min_pairs=33)
    path = tmp_path / "tune.txt"
    ia.write_tuning(t, str(path), header="a test table")
    assert path.read_text().startswith("# a test table\n")
    restore_table.setenv("INDIALIGN_TUNE_TABLE", str(path))
    ia.set_tuning(None)  # reload from the file
    assert ia.get_tuning() == t


def test_malformed_file_falls_back_to_built_in_rows(tmp_path, restore_table):
    path = tmp_path / "bad.txt"
    path.write_text("split 1\nbucket 0 max_len 128 bank_chunk 100 bank_cutoff_major 1 chain_chunk 16 "
                    "chain_smem_trace 1\n")  # bank_chunk not a multiple of 32
    restore_table.setenv("INDIALIGN_TUNE_TABLE", str(path))
    ia.set_tuning(None)
    got = ia.get_tuning()
    assert [r["max_len"] for r in got["rows"]] == [128, 512, 65535]
    assert all(r["bank_chunk"] == 256 for r in got["rows"])
    path.write_text("split 1\nnonsense line\n")
    ia.set_tuning(None)
    assert ia.get_tuning()["rows"][0]["bank_chunk"] == 256
    restore_table.setenv("INDIALIGN_TUNE_TABLE", str(tmp_path / "missing.txt"))
    ia.set_tuning(None)
    assert ia.get_tuning()["split"] == 0 and ia.get_tuning()["min_pairs"] == 64


@pytest.mark.parametrize("field,value", [("bank_chunk", 16), ("bank_chunk", 8192), ("bank_chunk", 100),
                                         ("bank_cutoff_major", 2), ("chain_chunk", 0), ("chain_chunk", 300),
                                         ("chain_smem_trace", 5), ("max_len", 0)])
def test_set_tuning_rejects_invalid_rows(field, value, restore_table):
    t = _table()
    t["rows"][1][field] = value
    with pytest.raises(ia.IndialignError, match="rc=-4"):
        ia.set_tuning(t)


def test_set_tuning_needs_ascending_buckets(restore_table):
    t = _table()
    t["rows"][1]["max_len"] = 50
    with pytest.raises(ia.IndialignError):
        ia.set_tuning(t)
    ok = copy.deepcopy(_table())
    ia.set_tuning(ok)
    assert ia.get_tuning() == ok


def test_shipped_table_parses():
    """The committed tune_b200.txt beside the library is a valid table."""
    import os
    path = os.path.join(os.path.dirname(ia.__file__), "tune_b200.txt")
    if not os.path.exists(path):
        pytest.skip("no tuned table committed")
    rows = [l.split() for l in open(path) if l.startswith("bucket")]
    assert len(rows) == ia.TUNE_BUCKETS
    for r in rows:
        kv = dict(zip(r[2::2], map(int, r[3::2])))
        assert set(kv) == set(ia.TUNE_FIELDS)
        assert kv["bank_chunk"] % 32 == 0 and 1 <= kv["chain_chunk"] <= 256
