"""The binary graph cache (the reference's Graph::writeToStream /
readFromStream format): byte parity with the reference's own writer (golden
digests from oracle/_ref, and live where the reference build exists), round
trips, and rejection of damaged files.  Host code only; no GPU."""
import hashlib
import json
import os
import subprocess

import numpy as np
import pytest

import asdmatch_b200 as A
import oracle_util as O
from asdmatch_b200 import workloads as W

HERE = os.path.dirname(os.path.abspath(__file__))


def _golden():
    with open(os.path.join(HERE, "golden", "binary_graph.json")) as fh:
        return json.load(fh)


@pytest.mark.parametrize("name,spec", [("c0", W.C0), ("c0d", W.C0D)])
def test_writer_matches_reference_digest(name, spec, tmp_path):
    g = W.graph(spec)
    p = str(tmp_path / "g.bin")
    g.write_binary(p)
    data = open(p, "rb").read()
    want = _golden()[name]
    assert len(data) == want["bytes"]
    assert hashlib.sha256(data).hexdigest() == want["sha256"]


@pytest.mark.skipif(not O.ref_available(), reason="needs oracle/_ref")
def test_writer_matches_live_reference_on_edge_cases(edge_files, tmp_path):
    for name, (q, qpath) in edge_files.items():
        ours, theirs = str(tmp_path / "o.bin"), str(tmp_path / "r.bin")
        q.write_binary(ours)
        subprocess.run([os.path.join(O.REF_DIR, "ref_count"), "-q", qpath, "-d", qpath, "-b", theirs], check=True,
                       capture_output=True)
        assert open(ours, "rb").read() == open(theirs, "rb").read(), name


def test_round_trip_keeps_the_csr(tmp_path):
    g = W.graph(W.C0)
    p = str(tmp_path / "g.bin")
    g.write_binary(p)
    h = A.HostGraph.load_binary(p)
    assert (h.n, h.m2, h.nlabels) == (g.n, g.m2, g.nlabels)
    assert np.array_equal(h.offsets, g.offsets)
    assert np.array_equal(h.nbrs, g.nbrs)
    assert np.array_equal(h.labels, g.labels)
    # and the loaded graph writes the same bytes again
    p2 = str(tmp_path / "g2.bin")
    h.write_binary(p2)
    assert open(p, "rb").read() == open(p2, "rb").read()


def test_damaged_files_are_rejected(tmp_path):
    g = W.graph(W.C0)
    p = str(tmp_path / "g.bin")
    g.write_binary(p)
    data = open(p, "rb").read()
    for bad in (data[:-4], data + b"\0\0\0\0", data[:10]):
        q = str(tmp_path / "bad.bin")
        open(q, "wb").write(bad)
        with pytest.raises(A.AsdmError) as e:
            A.HostGraph.load_binary(q)
        assert e.value.code == A.ERR_INVALID
    with pytest.raises(A.AsdmError) as e:
        A.HostGraph.load_binary(str(tmp_path / "missing.bin"))
    assert e.value.code == A.ERR_IO
