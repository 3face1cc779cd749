"""Generates tests/golden/golden.json from the reference implementation.

Run here, where the reference sources exist and oracle/ref.mk has built
oracle/_ref/{ref_count,ref_local,ref_embed}:

    make -f oracle/ref.mk && python tests/golden/make_golden.py

For every seeded synthetic query (asdmatch_b200/workloads.py) it records the
reference's exact count (ALL_LEVEL build), the SHA-256 of its candidate-space
dump (CandidateSpace::writeToStream plus the candidate sets), and for the
queries small enough to enumerate, the SHA-256 of its |Vg| x |Vq| LOCAL_COUNT
CSV and of its sorted embedding dump (storeMatches format).  The graphs and
queries themselves are not stored: every machine regenerates them from the
seeds with the product's generator, and the JSON pins the generator too (a
digest of each generated file).
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(HERE))

import asdmatch_b200 as A  # noqa: E402
import oracle_util as O  # noqa: E402
from asdmatch_b200 import workloads as W  # noqa: E402

EMBED_LIMIT = 200_000   # enumerate (CSV + embeddings) only below this many matches


def edge_case_queries():
    """Small hand-built queries exercising the corners of the candidate filter and the join."""
    cases = []
    # (name, n, labels, edges)
    cases.append(("edge", 2, [0, 0], [(0, 1)]))
    cases.append(("triangle", 3, [0, 0, 0], [(0, 1), (1, 2), (0, 2)]))
    cases.append(("path4_samelabel", 4, [1, 1, 1, 1], [(0, 1), (1, 2), (2, 3)]))
    cases.append(("star5", 5, [0, 1, 1, 1, 1], [(0, 1), (0, 2), (0, 3), (0, 4)]))
    cases.append(("square", 4, [0, 1, 0, 1], [(0, 1), (1, 2), (2, 3), (3, 0)]))
    cases.append(("diamond", 4, [0, 0, 1, 1], [(0, 1), (0, 2), (1, 2), (1, 3), (2, 3)]))
    cases.append(("absent_label", 3, [0, 0, 250], [(0, 1), (1, 2)]))
    cases.append(("bowtie", 5, [0, 1, 1, 2, 2], [(0, 1), (0, 2), (1, 2), (0, 3), (0, 4), (3, 4)]))
    cases.append(("k4", 4, [0, 0, 0, 0], [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]))
    return cases


def record(qpath, dpath, tmp, enumerate_all):
    rec = {}
    cs = os.path.join(tmp, "cs.txt")
    rec["count"] = O.ref_run("ref_count", qpath, dpath, cs=cs)
    rec["cs_sha"] = O.sha256_file(cs) if os.path.exists(cs) else None
    if os.path.exists(cs):
        os.remove(cs)
    if enumerate_all and rec["count"] <= EMBED_LIMIT:
        csv, emb = os.path.join(tmp, "l.csv"), os.path.join(tmp, "e.txt")
        for p in (csv, emb):
            if os.path.exists(p):
                os.remove(p)
        c2 = O.ref_run("ref_embed", qpath, dpath, csv=csv, emb=emb)
        assert c2 == rec["count"], (qpath, c2, rec["count"])
        # an empty candidate space ends the reference run before any output file
        if os.path.exists(csv):
            rec["csv_sha"] = O.sha256_file(csv)
            rec["emb_sha"] = O.sha256_file(emb)
    return rec


def main():
    if not O.ref_available():
        sys.exit("oracle/_ref is not built: make -f oracle/ref.mk")
    out = {"generator": {}, "sets": {}}
    with tempfile.TemporaryDirectory() as tmp:
        for name, spec, qseed, nq, sizes, n_enum in (("c0", W.C0, W.C0_QUERY_SEED, 200, [8], 40),
                                                     ("c0d", W.C0D, W.C0D_QUERY_SEED, 40, [6, 8], 24)):
            g = W.graph(spec)
            d = os.path.join(tmp, name)
            dpath, _ = W.write_workload(d, g, [])
            out["generator"][name] = {"spec": spec, "data_sha": O.sha256_file(dpath)}
            recs = []
            for size in sizes:
                qs = W.queries(g, size, nq, qseed + 100 * size)
                _, qpaths = W.write_workload(d, g, qs, prefix="s%d_" % size)
                for i, qp in enumerate(qpaths):
                    r = record(qp, dpath, tmp, i < n_enum)
                    r.update(size=size, index=i, seed=qseed + 100 * size + i, q_sha=O.sha256_file(qp))
                    recs.append(r)
                    print(name, size, i, r["count"], "enum" if "csv_sha" in r else "")
            out["sets"][name] = recs
        # edge cases on the config-0 graph
        g = W.graph(W.C0)
        dpath, _ = W.write_workload(os.path.join(tmp, "c0"), g, [])
        recs = []
        for cname, n, labels, edges in edge_case_queries():
            q = A.HostGraph.from_edges(n, labels, edges)
            qp = os.path.join(tmp, "edge_%s.graph" % cname)
            q.write(qp)
            r = record(qp, dpath, tmp, True)
            r.update(name=cname, n=n, labels=labels, edges=edges)
            recs.append(r)
            print("edge", cname, r["count"])
        out["sets"]["edge"] = recs
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
