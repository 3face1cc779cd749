"""GPU tests of the tree program: tree queries are counted by a bottom-up
program over the candidate edges instead of enumeration (with inclusion-
exclusion over same-label blocks when two non-adjacent vertices share a
label).  Its counts
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


def _adj(q):
    return [set(q.nbrs[q.offsets[u]:q.offsets[u + 1]].tolist()) for u in range(q.n)]


def tree_by_inclusion_exclusion(q):
    """True when every partition of each label's vertices into blocks of
    pairwise non-adjacent vertices has a tree as quotient (the tree program
    then counts the query by inclusion-exclusion)."""
    if q.m2 // 2 != q.n - 1:
        return False
    adj = _adj(q)
    labels = q.labels.tolist()
    ok = True

    def quotient_is_tree(block, nb):
        edges = {(min(block[u], block[w]), max(block[u], block[w])) for u in range(q.n) for w in adj[u]}
        return all(a != b for a, b in edges) and len(edges) == nb - 1

    def place(u, block, members):
        nonlocal ok
        if not ok:
            return
        if u == q.n:
            ok = quotient_is_tree(block, len(members))
            return
        for b, m in enumerate(members):
            if labels[m[0]] == labels[u] and not any(w in adj[u] for w in m):
                m.append(u)
                block[u] = b
                place(u + 1, block, members)
                m.pop()
        block[u] = len(members)
        members.append([u])
        place(u + 1, block, members)
        members.pop()

    place(0, [0] * q.n, [])
    return ok


def test_conflicted_trees_match_golden_and_enumeration(golden, c0_files):
    """Tree queries with same-label non-adjacent vertices: counted by the
    tree program's inclusion-exclusion (no root task runs) where every
    quotient is a tree, by enumeration otherwise; all match the golden counts
    and a LOCAL-mode enumeration of every match."""
    g, _, qs, _ = c0_files
    dg = A.DeviceGraph(g)
    by_program = 0
    for rec in golden["sets"]["c0"]:
        q = qs[rec["index"]]
        if q.m2 // 2 != q.n - 1 or conflict_free_tree(q):
            continue
        r = A.match(dg, q)
        assert r.count == rec["count"], rec["index"]
        if tree_by_inclusion_exclusion(q):
            assert r.tasks == 0, rec["index"]
            by_program += 1
            loc = A.match(dg, q, mode=A.MODE_LOCAL)  # enumeration
            assert int(loc.local_counts[:, 0].sum()) == rec["count"]
    dg.close()
    assert by_program >= 5


def _label_order(g):
    counts = np.bincount(g.labels.astype(np.int64))
    return np.argsort(-counts).tolist()


def test_conflicted_tree_shapes_against_oracle(c0d_files, dg_c0d, tmp_path):
    """Hand-made trees on the dense graph: same-label siblings (star with
    three equal leaves: blocks of three, coefficient +2), grandparent and
    grandchild of one label, two same-label pairs at once, a block of a
    vertex and two grandchildren, and same-label pairs at distance 3 or 4
    (quotients with a cycle: enumeration)."""
    g, dpath, _ = c0d_files
    L = _label_order(g)
    a, b, c = L[0], L[1], L[2]
    shapes = [
        ("star3", 4, [a, b, b, b], [(0, 1), (0, 2), (0, 3)]),
        ("star4", 5, [a, b, b, b, c], [(0, 1), (0, 2), (0, 3), (0, 4)]),
        ("path_gp", 4, [a, b, a, c], [(0, 1), (1, 2), (2, 3)]),
        ("path_two_pairs", 4, [a, b, a, b], [(0, 1), (1, 2), (2, 3)]),
        ("spider", 6, [a, b, b, a, a, c], [(0, 1), (0, 2), (1, 3), (1, 4), (0, 5)]),
        ("path_d3", 4, [a, b, c, a], [(0, 1), (1, 2), (2, 3)]),
        ("all_one_label_path", 5, [a, a, a, a, a], [(0, 1), (1, 2), (2, 3), (3, 4)]),
    ]
    qs = [A.HostGraph.from_edges(n, lab, e) for _, n, lab, e in shapes]
    counts, status = A.run_batch(dg_c0d, qs)
    for (name, *_), q, cnt, st in zip(shapes, qs, counts.tolist(), status.tolist()):
        qp = str(tmp_path / (name + ".graph"))
        q.write(qp)
        want, _ = O.oracle_run(qp, dpath, O.MODE_COUNT)
        assert st == 0 and cnt == want, name
        r = A.match(dg_c0d, q)
        assert r.count == want, name
        if tree_by_inclusion_exclusion(q):
            assert r.tasks == 0, name
        else:
            assert name in ("path_d3", "all_one_label_path"), name
    assert tree_by_inclusion_exclusion(qs[0]) and not tree_by_inclusion_exclusion(qs[5])
