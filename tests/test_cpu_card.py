"""The .card plan cache reader/writer (host code only)."""
import os
import tarfile

import pytest

import asdmatch_b200 as A
import oracle_util as O

YEAST = O.reference_file("dataset", "yeast.tar.gz")


def test_write_then_read_round_trip(tmp_path):
    c = A.Card()
    c[0b11] = 12.345        # values keep two decimals, like saveSubsetToCard
    c[0b101] = 7
    c[0b111] = 1e12
    p = str(tmp_path / "x.card")
    c.write(p, plan_seconds=1.25)
    d = A.Card(p)
    assert d.info() == {"bags": 0, "entries": 3, "plan_seconds": 1.25}
    assert d[0b11] == 12.34 and d[0b101] == 7.0 and d[0b111] == 1e12
    with pytest.raises(A.AsdmError):
        d[0b1000]


def test_garbage_and_missing_files_are_rejected(tmp_path):
    p = tmp_path / "bad.card"
    p.write_bytes(b"\x01\x02\x03")
    with pytest.raises(A.AsdmError) as e:
        A.Card(str(p))
    assert e.value.code == A.ERR_INVALID
    with pytest.raises(A.AsdmError) as e:
        A.Card(str(tmp_path / "none.card"))
    assert e.value.code == A.ERR_IO


@pytest.mark.skipif(not YEAST, reason="needs the reference's yeast fixtures")
def test_reads_the_reference_card_files(tmp_path):
    with tarfile.open(YEAST) as t:
        t.extractall(tmp_path)
    qdir = tmp_path / "yeast" / "query_graph"
    cards = sorted(p for p in os.listdir(qdir) if p.endswith(".card"))
    assert len(cards) == 1000
    for name in cards:
        c = A.Card(str(qdir / name))
        info = c.info()
        n = int(name.split("_")[1])
        assert info["bags"] >= 1 and info["entries"] > 0, name
        # every key is a subset of the query's vertex set
        assert info["plan_seconds"] >= 0
    c = A.Card(str(qdir / "query_8_1.card"))
    assert all(0 < k < (1 << 8) for k in [1, 2, 4]) and c.info()["entries"] > 0
