"""Parity on the config-4 graph (N=1.0M, M=10M, 32 labels), against the
reference's own outputs at the graph's full size (tests/golden/c4_batch.json,
made by tests/golden/make_c4_golden.py):
* the |Vg| x |Vq| LOCAL_COUNT matrix of every "parity" query the reference
  finished (random-walk queries of 4..8 vertices) against the SHA-256 of the
  reference's CSV (oracle/_ref/ref_local, written by main.cpp:135-146),
  batched and one query at a time;
* the sorted embedding set of every "embed" query the reference finished
  (dense random-walk queries of 5..8 vertices) against the SHA-256 of the
  reference's storeMatches dump (oracle/_ref/ref_embed,
  matching/join.cpp:1099-1107).
"""
import hashlib
import io
import json
import os

import numpy as np
import pytest

import asdmatch_b200 as A
from asdmatch_b200 import workloads as W

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c4_batch.json")


def csv_sha(local):
    """SHA-256 of the CSV text the reference writes for a local-count matrix:
    one row per data vertex, values joined by commas.  Rows of zeros are
    hashed as one repeated string, so a 1M-row matrix costs only its nonzero rows."""
    h = hashlib.sha256()
    nq = local.shape[1]
    zero = (",".join(["0"] * nq) + "\n").encode()
    prev = 0
    for r in np.flatnonzero(local.any(axis=1)).tolist():
        if r > prev:
            h.update(zero * (r - prev))
        h.update((",".join(str(int(x)) for x in local[r]) + "\n").encode())
        prev = r + 1
    if local.shape[0] > prev:
        h.update(zero * (local.shape[0] - prev))
    return h.hexdigest()


def emb_sha(emb):
    """SHA-256 of the reference's storeMatches text for a sorted embedding
    set: the row count, then one row per embedding, each value followed by a space."""
    buf = io.BytesIO()
    buf.write(b"%d\n" % len(emb))
    if len(emb):
        np.savetxt(buf, emb, fmt="%d ", delimiter="", newline="\n")
    return hashlib.sha256(buf.getvalue()).hexdigest()


@pytest.fixture(scope="module")
def c4_graph():
    g = W.graph(W.C4)
    dg = A.DeviceGraph(g)
    with open(GOLDEN) as fh:
        data = json.load(fh)
    yield g, dg, data
    dg.close()


@pytest.fixture(scope="module")
def c4(c4_graph):
    g, dg, data = c4_graph
    recs = [r for r in data["parity"] if r["count"] is not None]
    specs = W.c4_parity_specs()
    qs = [W.from_specs(g, [specs[r["index"]]])[0] for r in recs]
    return dg, recs, qs


def test_batched_local_counts_match_reference_csv(c4):
    dg, recs, qs = c4
    assert len(recs) >= 10 and len({r["size"] for r in recs}) >= 3
    for k in range(0, len(recs), 8):
        counts, status, mats = A.run_batch_local(dg, qs[k:k + 8])
        for r, c, st, m in zip(recs[k:k + 8], counts.tolist(), status.tolist(), mats):
            assert st == A.OK and c == r["count"], (r["index"], st, c, r["count"])
            assert csv_sha(m) == r["csv_sha256"], r["index"]


def test_single_query_local_counts_match_reference_csv(c4):
    dg, recs, qs = c4
    # one of each size, heaviest first
    seen = set()
    for r, q in sorted(zip(recs, qs), key=lambda t: -t[0]["count"]):
        if r["size"] in seen:
            continue
        seen.add(r["size"])
        res = A.match(dg, q, mode=A.MODE_LOCAL)
        assert res.count == r["count"], r["index"]
        assert csv_sha(res.local_counts) == r["csv_sha256"], r["index"]
    assert len(seen) >= 3


def test_embeddings_match_reference_dump(c4_graph):
    g, dg, data = c4_graph
    recs = [r for r in data["embed"] if r["count"] is not None and r["count"] <= 5_000_000]
    assert len(recs) >= 4 and len({r["size"] for r in recs}) >= 2
    for r in recs:
        q = W.from_specs(g, [(r["size"], r["seed"], r["density"])])[0]
        res = A.match(dg, q, mode=A.MODE_EMBED)
        assert res.count == r["count"] == len(res.embeddings), r["index"]
        assert emb_sha(res.embeddings) == r["emb_sha256"], r["index"]
