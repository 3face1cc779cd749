"""GPU tests of the count lower bound (asdm_cs_count_lower_bound) that lets
the counting entry points report ASDM_ERR_OVERFLOW for counts of 2^64 and
more without enumerating them.

The bound counts a subset of the embeddings (same-label query vertices on
disjoint hash classes of candidates, a feedback vertex set fixed to hubs), so
it may never exceed the exact count: that is checked against the golden
reference counts.  On graphs built so that the exact count is known in closed
form and lies far above 2^64, the bound must prove the overflow, and every
counting entry point must then report ASDM_ERR_OVERFLOW."""
import math

import numpy as np
import pytest

import asdmatch_b200 as A

pytestmark = pytest.mark.gpu

TWO64 = 1 << 64


def test_lower_bound_never_exceeds_golden_counts(golden, c0_files, c0d_files):
    checked, positive = 0, 0
    for g, recs, qs in ((c0_files[0], golden["sets"]["c0"], c0_files[2]),
                        (c0d_files[0], golden["sets"]["c0d"], None)):
        dg = A.DeviceGraph(g)
        for k, rec in enumerate(recs):
            if qs is not None:
                q = qs[rec["index"]]
            else:
                q = g.random_walk_query(rec["size"], rec["seed"], 0)
            cs = A.CandidateSpace(dg, q)
            lb, exceeds = cs.count_lower_bound()
            cs.close()
            assert not exceeds and lb <= rec["count"], (k, lb, rec["count"])
            checked += 1
            positive += lb > 0
        dg.close()
    assert checked == 280
    assert positive >= 20  # the bound is not trivially zero


def _star_graph(leaves):
    # hub 0 (label 0) joined to `leaves` vertices of label 1
    n = leaves + 1
    labels = [0] + [1] * leaves
    edges = [(0, 1 + i) for i in range(leaves)]
    return A.HostGraph.from_edges(n, labels, edges)


def _book_graph(pages):
    # hub 0 (label 0) and spine 1 (label 2) joined, each page vertex (label 1) joined to both
    n = pages + 2
    labels = [0, 2] + [1] * pages
    edges = [(0, 1)] + [(0, 2 + i) for i in range(pages)] + [(1, 2 + i) for i in range(pages)]
    return A.HostGraph.from_edges(n, labels, edges)


def _falling(n, k):
    return math.prod(range(n - k + 1, n + 1))


@pytest.mark.parametrize("kind", ["star", "book"])
def test_overflow_is_proven_where_the_count_is_known(kind):
    if kind == "star":
        big, k = 3000, 9
        g = _star_graph(big)
        q = A.HostGraph.from_edges(k + 1, [0] + [1] * k, [(0, 1 + i) for i in range(k)])
    else:
        big, k = 6000, 8
        g = _book_graph(big)
        q = A.HostGraph.from_edges(k + 2, [0, 2] + [1] * k,
                                   [(0, 1)] + [(0, 2 + i) for i in range(k)] + [(1, 2 + i) for i in range(k)])
    exact = _falling(big, k)  # the k same-label query vertices take distinct data vertices
    assert exact >= TWO64
    dg = A.DeviceGraph(g)
    cs = A.CandidateSpace(dg, q)
    lb, exceeds = cs.count_lower_bound()
    assert exceeds and lb == TWO64 - 1
    with pytest.raises(A.AsdmError) as e:
        A.adaptive_share_join(cs)
    assert e.value.code == A.ERR_OVERFLOW
    cs.close()
    counts, status = A.run_batch(dg, [q, q])
    assert status.tolist() == [A.ERR_OVERFLOW] * 2
    dg.close()


def test_lower_bound_below_two64_is_exact_on_small_known_counts():
    # the same shapes with small sizes: the bound is a lower bound of the exact count
    g = _book_graph(40)
    dg = A.DeviceGraph(g)
    for k in (2, 3, 4):
        q = A.HostGraph.from_edges(k + 2, [0, 2] + [1] * k,
                                   [(0, 1)] + [(0, 2 + i) for i in range(k)] + [(1, 2 + i) for i in range(k)])
        cs = A.CandidateSpace(dg, q)
        lb, exceeds = cs.count_lower_bound()
        exact = _falling(40, k)
        assert not exceeds and 0 < lb <= exact
        assert A.adaptive_share_join(cs).count == exact
        cs.close()
    dg.close()


def _far_pairs(q):
    """Same-label pairs three or more edges apart."""
    adj = [set(q.nbrs[q.offsets[u]:q.offsets[u + 1]].tolist()) for u in range(q.n)]
    far = []
    for a in range(q.n):
        dist = {a: 0}
        frontier = [a]
        while frontier:
            nxt = []
            for x in frontier:
                for y in adj[x]:
                    if y not in dist:
                        dist[y] = dist[x] + 1
                        nxt.append(y)
            frontier = nxt
        far += [(a, b) for b in range(a + 1, q.n) if q.labels[a] == q.labels[b] and dist.get(b, 99) >= 3]
    return far


def test_tree_bound_is_the_exact_count_without_far_pairs(golden, c0_files, c0d_files):
    """For a tree query whose same-label vertices are all two edges apart the
    tree bound restricts nothing: it is the inclusion-exclusion count itself,
    exact in doubles below 2^53; with far pairs it stays a lower bound."""
    exact_checked = below = 0
    for g, recs, qs in ((c0_files[0], golden["sets"]["c0"], c0_files[2]),
                        (c0d_files[0], golden["sets"]["c0d"], None)):
        dg = A.DeviceGraph(g)
        for rec in recs:
            q = qs[rec["index"]] if qs is not None else g.random_walk_query(rec["size"], rec["seed"], 0)
            if q.m2 // 2 != q.n - 1 or rec["count"] == 0:
                continue
            cs = A.CandidateSpace(dg, q)
            lb, exceeds = cs.count_lower_bound()
            cs.close()
            assert not exceeds
            if not _far_pairs(q):
                assert lb == rec["count"], (rec["index"], lb, rec["count"])
                exact_checked += 1
            else:
                assert lb <= rec["count"]
                below += 1
        dg.close()
    assert exact_checked >= 30 and below >= 1, (exact_checked, below)


def _broom_graph(m, p):
    # hub 0 (label 0) joined to m vertices of label 2, each joined to p vertices of label 1 of its own
    n = 1 + m + m * p
    labels = [0] + [2] * m + [1] * (m * p)
    edges = [(0, 1 + i) for i in range(m)]
    edges += [(1 + i, 1 + m + i * p + j) for i in range(m) for j in range(p)]
    return A.HostGraph.from_edges(n, labels, edges)


def _broom_query(k):
    # centre (label 0), k children (label 2), one leaf (label 1) under each: the leaves are four edges apart
    labels = [0] + [2] * k + [1] * k
    edges = [(0, 1 + i) for i in range(k)] + [(1 + i, 1 + k + i) for i in range(k)]
    return A.HostGraph.from_edges(2 * k + 1, labels, edges)


def test_pair_bound_proves_what_classes_cannot():
    """Brooms: the exact count falling(m, 4) * p^4 = 1.55e21 is above 2^64,
    but a bound that keeps the four far-apart leaves on four hash classes of
    candidates keeps about 1/256 of it (6e18, below 2^64).  The first-order
    pair bound (homomorphisms minus those that join a same-label pair) loses
    only a few percent and proves the overflow; on a small broom it stays
    below the exact count."""
    m, p, k = 200, 1000, 4
    exact = _falling(m, k) * p ** k
    assert exact >= TWO64 and exact // 256 < TWO64
    dg = A.DeviceGraph(_broom_graph(m, p))
    q = _broom_query(k)
    cs = A.CandidateSpace(dg, q)
    lb, exceeds = cs.count_lower_bound()
    cs.close()
    assert exceeds and lb == TWO64 - 1
    counts, status = A.run_batch(dg, [q])
    assert status.tolist() == [A.ERR_OVERFLOW]
    dg.close()
    m, p = 40, 30
    dg = A.DeviceGraph(_broom_graph(m, p))
    cs = A.CandidateSpace(dg, q)
    lb, exceeds = cs.count_lower_bound()
    exact = _falling(m, k) * p ** k
    # H = m^4 p^4, minus 6 merged sibling pairs (m^3 p^4 each) and 6 merged leaf pairs (m^4 p^3 each)
    want = m ** 4 * p ** 4 - 6 * m ** 3 * p ** 4 - 6 * m ** 4 * p ** 3
    assert not exceeds and want * (1 - 1e-12) <= lb <= exact, (lb, want, exact)
    assert A.adaptive_share_join(cs).count == exact
    cs.close()
    dg.close()
