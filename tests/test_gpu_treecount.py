"""GPU tests of the tree program: conflict-free tree queries are counted by a
bottom-up program over the candidate edges instead of enumeration.  Its counts
are checked against the golden reference counts, against the enumeration path
(LOCAL mode walks every match) and against the CPU oracle, in the single-query
and batched forms."""
import numpy as np
import pytest

import asdmatch_b200 as A
import oracle_util as O
from asdmatch_b200 import workloads as W

pytestmark = pytest.mark.gpu


def conflict_free_tree(q):
    if q.m2 // 2 != q.n - 1:
        return False
    adj = [set(q.nbrs[q.offsets[u]:q.offsets[u + 1]].tolist()) for u in range(q.n)]
    return not any(q.labels[u] == q.labels[w] and w not in adj[u] for u in range(q.n) for w in range(u + 1, q.n))


@pytest.fixture(scope="module")
def dg_c0d(c0d_files):
    dg = A.DeviceGraph(c0d_files[0])
    yield dg
    dg.close()


def test_tree_program_matches_golden_and_enumeration(golden, c0_files):
    g, _, qs, _ = c0_files
    dg = A.DeviceGraph(g)
    checked = 0
    for rec in golden["sets"]["c0"]:
        q = qs[rec["index"]]
        if not conflict_free_tree(q):
            continue
        r = A.match(dg, q)
        assert r.count == rec["count"], rec["index"]
        loc = A.match(dg, q, mode=A.MODE_LOCAL)  # enumerates every match
        assert int(loc.local_counts[:, 0].sum()) == rec["count"]
        checked += 1
    dg.close()
    assert checked >= 30


def test_tree_program_on_denser_trees_against_oracle(c0d_files, dg_c0d, tmp_path):
    g, dpath, _ = c0d_files
    trees = []
    for seed in range(20000, 24000):
        q = g.random_walk_query(4 + seed % 3, seed, 2)
        if conflict_free_tree(q):
            trees.append(q)
        if len(trees) == 24:
            break
    assert len(trees) >= 12
    counts, status = A.run_batch(dg_c0d, trees)
    assert status.tolist() == [0] * len(trees)
    assert counts.sum() > 0
    for q, c in zip(trees, counts.tolist()):
        qp = str(tmp_path / "q.graph")
        q.write(qp)
        want, _ = O.oracle_run(qp, dpath, O.MODE_COUNT)
        assert c == want
        assert A.match(dg_c0d, q).count == want
        loc = A.match(dg_c0d, q, mode=A.MODE_LOCAL)
        assert int(loc.local_counts[:, 0].sum()) == want


def _csv_matrix(path, n):
    rows = [list(map(int, line.split(","))) for line in open(path) if line.strip()]
    return np.asarray(rows, dtype=np.uint64).reshape(-1, n)


def test_tree_program_local_counts_against_oracle_csv(c0d_files, dg_c0d, tmp_path):
    g, dpath, _ = c0d_files
    trees = []
    for seed in range(30000, 34000):
        q = g.random_walk_query(4 + seed % 4, seed, 2)
        if conflict_free_tree(q):
            trees.append(q)
        if len(trees) == 10:
            break
    assert len(trees) >= 6
    counts, status, mats = A.run_batch_local(dg_c0d, trees)
    assert status.tolist() == [0] * len(trees)
    for q, c, m in zip(trees, counts.tolist(), mats):
        qp, csv = str(tmp_path / "q.graph"), str(tmp_path / "l.csv")
        q.write(qp)
        want, _ = O.oracle_run(qp, dpath, O.MODE_LOCAL, csv=csv)
        assert c == want
        ref = _csv_matrix(csv, q.n)
        assert np.array_equal(m, ref)
        single = A.match(dg_c0d, q, mode=A.MODE_LOCAL)
        assert single.count == want and np.array_equal(single.local_counts, ref)
