"""The CPU oracle against the reference's golden vectors (and, where the
reference build exists in this container, against the reference live)."""
import os

import pytest

import oracle_util as O

YEAST = O.reference_file("dataset", "yeast.tar.gz")


def _check(rec, qpath, dpath, tmp_path, full):
    cs = str(tmp_path / "cs.txt")
    csv = str(tmp_path / "l.csv") if full else None
    emb = str(tmp_path / "e.txt") if full else None
    mode = O.MODE_EMBED if full else O.MODE_COUNT
    count, flags = O.oracle_run(qpath, dpath, mode, csv=csv, emb=emb, cs=cs)
    assert count == rec["count"], qpath
    if rec.get("cs_sha") is not None and rec["count"] > 0:
        assert O.sha256_file(cs) == rec["cs_sha"], qpath
    if full:
        assert O.sha256_file(csv) == rec["csv_sha"], qpath
        assert O.sha256_file(emb) == rec["emb_sha"], qpath


def test_oracle_c0_counts_and_candidate_spaces(golden, c0_files, tmp_path):
    _, dpath, _, qpaths = c0_files
    for rec in golden["sets"]["c0"]:
        _check(rec, qpaths[rec["index"]], dpath, tmp_path, "csv_sha" in rec)


def test_oracle_c0d(golden, c0d_files, tmp_path):
    _, dpath, by_size = c0d_files
    for rec in golden["sets"]["c0d"]:
        if rec["count"] > 3_000_000 and "csv_sha" not in rec:
            continue  # keep the CPU suite short; the GPU suite covers these
        _check(rec, by_size[rec["size"]][1][rec["index"]], dpath, tmp_path, "csv_sha" in rec)


def test_oracle_edge_cases(golden, c0_files, edge_files, tmp_path):
    _, dpath, _, _ = c0_files
    for rec in golden["sets"]["edge"]:
        _check(rec, edge_files[rec["name"]][1], dpath, tmp_path, "csv_sha" in rec)


@pytest.mark.skipif(not (YEAST and O.ref_available()), reason="needs the reference tree and oracle/_ref")
def test_oracle_matches_reference_on_yeast(tmp_path):
    import tarfile
    with tarfile.open(YEAST) as t:
        t.extractall(tmp_path)
    base = tmp_path / "yeast"
    dpath = str(base / "data_graph" / "yeast.graph")
    for size, idx in ((8, range(1, 21)), (12, range(1, 6)), (16, range(1, 4))):
        for i in idx:
            q = str(base / "query_graph" / ("query_%d_%d.graph" % (size, i)))
            rcs, ocs = str(tmp_path / "r.txt"), str(tmp_path / "o.txt")
            r = O.ref_run("ref_count", q, dpath, cs=rcs)
            c, _ = O.oracle_run(q, dpath, O.MODE_COUNT, cs=ocs)
            assert c == r, q
            assert O.sha256_file(rcs) == O.sha256_file(ocs), q


def test_oracle_tree_count_matches_golden_counts(golden, c0_files, tmp_path):
    """The oracle's inclusion-exclusion tree count (asdm_oracle -t) equals the
    reference's count on every config-0 tree query it can count this way."""
    import subprocess
    g, dpath, qs, qpaths = c0_files
    O.build_oracle()
    recs = [r for r in golden["sets"]["c0"] if qs[r["index"]].m2 // 2 == qs[r["index"]].n - 1]
    lst = tmp_path / "trees.txt"
    lst.write_text("\n".join(qpaths[r["index"]] for r in recs) + "\n")
    out = subprocess.run([O.ORACLE_BIN, "-d", dpath, "-t", str(lst)], capture_output=True, text=True, check=True)
    counted = 0
    for line in out.stdout.splitlines():
        _, k, st, *rest = line.split()
        rec = recs[int(k)]
        if st == "ok":
            assert int(rest[0]) == rec["count"], rec["index"]
            counted += 1
        else:
            assert st in ("skip", "empty") and (st == "skip" or rec["count"] == 0), (rec["index"], st)
    assert counted >= 30


def test_oracle_lower_bound_never_exceeds_golden_counts(golden, c0_files, tmp_path):
    """The oracle's restatement of the device's overflow lower bound (asdm_oracle
    -b) counts a subset of the embeddings: never more than the reference's count."""
    import subprocess
    g, dpath, qs, qpaths = c0_files
    O.build_oracle()
    recs = golden["sets"]["c0"]
    lst = tmp_path / "all.txt"
    lst.write_text("\n".join(qpaths[r["index"]] for r in recs) + "\n")
    out = subprocess.run([O.ORACLE_BIN, "-d", dpath, "-b", str(lst)], capture_output=True, text=True, check=True)
    formed = positive = 0
    for line in out.stdout.splitlines():
        _, k, v = line.split()
        rec = recs[int(k)]
        if v in ("none", "empty"):
            continue
        formed += 1
        assert int(v) <= rec["count"], (rec["index"], v, rec["count"])
        positive += int(v) > 0
    assert formed >= 150 and positive >= 20


def _far_same_label_pair(q):
    """Whether tree query q has two same-label vertices three or more edges apart."""
    off, nb, lab = q.offsets, q.nbrs, q.labels
    for r in range(q.n):
        dist = {r: 0}
        front = [r]
        for u in front:
            for e in range(off[u], off[u + 1]):
                w = int(nb[e])
                if w not in dist:
                    dist[w] = dist[u] + 1
                    front.append(w)
        if any(w != r and lab[w] == lab[r] and d >= 3 for w, d in dist.items()):
            return True
    return False


def test_oracle_tree_bound_is_the_count_without_far_pairs(golden, c0_files, tmp_path):
    """For a tree whose same-label vertices are all within two edges, the
    far-class tree bound restricts nothing: asdm_oracle -b gives the exact
    count, equal to the reference's."""
    import subprocess
    g, dpath, qs, qpaths = c0_files
    O.build_oracle()
    recs = [r for r in golden["sets"]["c0"]
            if qs[r["index"]].m2 // 2 == qs[r["index"]].n - 1 and not _far_same_label_pair(qs[r["index"]])]
    lst = tmp_path / "near.txt"
    lst.write_text("\n".join(qpaths[r["index"]] for r in recs) + "\n")
    out = subprocess.run([O.ORACLE_BIN, "-d", dpath, "-b", str(lst)], capture_output=True, text=True, check=True)
    equal = 0
    for line in out.stdout.splitlines():
        _, k, v = line.split()
        rec = recs[int(k)]
        if v == "empty":
            assert rec["count"] == 0
            continue
        assert int(v) == rec["count"], (rec["index"], v, rec["count"])
        equal += 1
    assert equal >= 40, (equal, len(recs))


def test_oracle_matches_reference_on_the_config4_graph(tmp_path):
    """At the config-4 graph's full size (1M vertices, 10M edges): the oracle's
    local-count CSVs and sorted embedding dumps equal the reference's
    (tests/golden/c4_batch.json, made with oracle/_ref) on the smallest
    finished queries of the parity and embed sets."""
    import json
    from asdmatch_b200 import workloads as W
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c4_batch.json")) as fh:
        data = json.load(fh)
    g = W.graph(W.C4)
    dpath = str(tmp_path / "data.graph")
    g.write(dpath)
    specs = W.c4_parity_specs()
    parity = sorted((r for r in data["parity"] if r["count"] is not None), key=lambda r: r["count"])[:2]
    embed = sorted((r for r in data["embed"] if r["count"] is not None), key=lambda r: r["count"])[:2]
    for r in parity:
        qpath = str(tmp_path / "p.graph")
        W.from_specs(g, [specs[r["index"]]])[0].write(qpath)
        csv = str(tmp_path / "l.csv")
        count, _ = O.oracle_run(qpath, dpath, O.MODE_LOCAL, csv=csv)
        assert count == r["count"] and O.sha256_file(csv) == r["csv_sha256"], r["index"]
    for r in embed:
        qpath = str(tmp_path / "e.graph")
        W.from_specs(g, [(r["size"], r["seed"], r["density"])])[0].write(qpath)
        emb = str(tmp_path / "e.txt")
        count, _ = O.oracle_run(qpath, dpath, O.MODE_EMBED, emb=emb)
        assert count == r["count"] and O.sha256_file(emb) == r["emb_sha256"], r["index"]


def test_oracle_counts_match_reference_on_the_config1_graph(tmp_path):
    """At the config-1 graph's full size (3.77M vertices, 16.5M edges): the
    oracle's backtracking count equals the reference's (tests/golden/c2_batch.json,
    made with oracle/_ref) on the two config-2 queries with the smallest
    reference counts, one of them outside the tree program's reach."""
    import json
    from asdmatch_b200 import workloads as W
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_batch.json")) as fh:
        data = json.load(fh)
    recs = sorted((r for r in data["queries"] if r.get("count") is not None), key=lambda r: r["count"])[:2]
    g = W.graph(W.C1)
    dpath = str(tmp_path / "data.graph")
    g.write(dpath)
    for r in recs:
        qpath = str(tmp_path / "q.graph")
        W.c2_candidate(g, r["index"])[2].write(qpath)
        count, _ = O.oracle_run(qpath, dpath, O.MODE_COUNT)
        assert count == r["count"], r["index"]
