"""GPU parity: the device candidate space, counts, local-count CSVs and
embedding sets against the reference's golden vectors, plus the
size-independent properties (plan invariance, consistency between modes)."""
import hashlib

import numpy as np
import pytest

import asdmatch_b200 as A

pytestmark = pytest.mark.gpu


def csv_sha(local):
    text = "".join(",".join(str(int(x)) for x in row) + "\n" for row in local)
    return hashlib.sha256(text.encode()).hexdigest()


def emb_sha(emb):
    text = "%d\n" % len(emb) + "".join("".join("%d " % int(x) for x in row) + "\n" for row in emb)
    return hashlib.sha256(text.encode()).hexdigest()


@pytest.fixture(scope="module")
def dg_c0(c0_files):
    dg = A.DeviceGraph(c0_files[0])
    yield dg
    dg.close()


@pytest.fixture(scope="module")
def dg_c0d(c0d_files):
    dg = A.DeviceGraph(c0d_files[0])
    yield dg
    dg.close()


def test_candidate_space_matches_reference_dump(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    for rec in golden["sets"]["c0"][:80]:
        cs = A.CandidateSpace(dg_c0, qs[rec["index"]])
        if rec["cs_sha"] is None:
            assert not cs.build_cand_cfl()
            continue
        assert cs.build_cand_cfl()
        assert hashlib.sha256(cs.write_to_stream().encode()).hexdigest() == rec["cs_sha"], rec["index"]
        cs.close()


def test_candidate_space_c0d(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    for rec in golden["sets"]["c0d"][::4]:
        cs = A.CandidateSpace(dg_c0d, by_size[rec["size"]][0][rec["index"]])
        assert hashlib.sha256(cs.write_to_stream().encode()).hexdigest() == rec["cs_sha"], rec
        cs.close()


def test_counts_c0(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    for rec in golden["sets"]["c0"]:
        assert A.match(dg_c0, qs[rec["index"]]).count == rec["count"], rec["index"]


def test_counts_c0d(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    for rec in golden["sets"]["c0d"]:
        assert A.match(dg_c0d, by_size[rec["size"]][0][rec["index"]]).count == rec["count"], rec


def test_local_counts_and_embeddings_c0(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    checked = 0
    for rec in golden["sets"]["c0"]:
        if "csv_sha" not in rec:
            continue
        r = A.match(dg_c0, qs[rec["index"]], mode=A.MODE_LOCAL | A.MODE_EMBED)
        assert r.count == rec["count"]
        assert csv_sha(r.local_counts) == rec["csv_sha"], rec["index"]
        assert emb_sha(r.embeddings) == rec["emb_sha"], rec["index"]
        checked += 1
    assert checked >= 30


def test_local_counts_and_embeddings_c0d(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    for rec in golden["sets"]["c0d"]:
        if "csv_sha" not in rec:
            continue
        r = A.match(dg_c0d, by_size[rec["size"]][0][rec["index"]], mode=A.MODE_LOCAL | A.MODE_EMBED)
        assert csv_sha(r.local_counts) == rec["csv_sha"], rec
        assert emb_sha(r.embeddings) == rec["emb_sha"], rec


def test_edge_cases(golden, dg_c0, edge_files):
    for rec in golden["sets"]["edge"]:
        q = edge_files[rec["name"]][0]
        r = A.match(dg_c0, q, mode=A.MODE_LOCAL | A.MODE_EMBED)
        assert r.count == rec["count"], rec["name"]
        if "csv_sha" in rec:
            assert csv_sha(r.local_counts) == rec["csv_sha"], rec["name"]
            assert emb_sha(r.embeddings) == rec["emb_sha"], rec["name"]


def _random_connected_order(q, rng):
    n = q.n
    start = int(rng.integers(n))
    order, seen = [start], {start}
    while len(order) < n:
        frontier = sorted({int(w) for u in order for w in q.nbrs[q.offsets[u]:q.offsets[u + 1]]} - seen)
        nxt = frontier[int(rng.integers(len(frontier)))]
        order.append(nxt)
        seen.add(nxt)
    return order


def test_count_is_plan_invariant(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    rng = np.random.default_rng(5)
    for rec in golden["sets"]["c0d"][40:56]:
        q = by_size[rec["size"]][0][rec["index"]]
        for _ in range(3):
            order = _random_connected_order(q, rng)
            assert A.match(dg_c0d, q, order=order).count == rec["count"], (rec, order)


def test_local_count_columns_sum_to_count(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    for rec in golden["sets"]["c0d"][40:50]:
        r = A.match(dg_c0d, by_size[rec["size"]][0][rec["index"]], mode=A.MODE_LOCAL)
        assert r.count == rec["count"]
        assert all(int(s) == rec["count"] for s in r.local_counts.sum(axis=0, dtype=np.uint64))


def test_count_query_and_batch_entry_points(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    recs = golden["sets"]["c0"][:50]
    for rec in recs[:10]:
        assert A.count_query(dg_c0, qs[rec["index"]]).count == rec["count"]
    counts, status = A.run_batch(dg_c0, [qs[r["index"]] for r in recs])
    assert status.tolist() == [0] * len(recs)
    assert counts.tolist() == [r["count"] for r in recs]


def test_leapfrog_join_matches_numpy():
    rng = np.random.default_rng(0)
    sets = []
    for k in (1, 2, 3, 5, 8, 31):
        for ratio in (1, 10, 1000):
            lists = []
            for j in range(k):
                n = int(rng.integers(0, 50)) * (ratio if j == 0 else 1) + (1 if j else 0)
                lists.append(np.unique(rng.integers(0, 4000, size=n)).astype(np.uint32))
            sets.append(lists)
    # long lists of similar length (merged over many 32-entry windows) and
    # lopsided ones (galloped); equal, interleaved and disjoint lists
    for k, n0, n1, span in ((2, 3000, 2500, 9000), (3, 700, 5000, 20000), (2, 40, 9000, 100000),
                            (4, 1500, 1600, 4000)):
        sets.append([np.unique(rng.integers(0, span, size=n0 if j == 0 else n1)).astype(np.uint32)
                     for j in range(k)])
    sets.append([np.arange(0, 4000, 2, dtype=np.uint32), np.arange(1, 4001, 2, dtype=np.uint32)])
    sets.append([np.arange(5000, dtype=np.uint32)] * 3)
    sets.append([np.arange(0, 3000, dtype=np.uint32), np.arange(3000, 6000, dtype=np.uint32)])
    sets.append([np.zeros(0, np.uint32), np.arange(10, dtype=np.uint32)])
    sets.append([])
    out = A.leapfrog_join(sets)
    for lists, got in zip(sets, out):
        if not lists:
            assert len(got) == 0
            continue
        want = lists[0]
        for l in lists[1:]:
            want = np.intersect1d(want, l)
        assert np.array_equal(got, want)


def test_time_limit_returns_status_and_device_stays_usable(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    rec = max(golden["sets"]["c0d"], key=lambda r: r["count"])
    q = by_size[rec["size"]][0][rec["index"]]
    with pytest.raises(A.AsdmError) as e:
        A.match(dg_c0d, q, time_limit_s=1e-7)
    assert e.value.code == A.ERR_TIMEOUT
    assert A.match(dg_c0d, q).count == rec["count"]


def test_bad_queries_are_rejected(dg_c0):
    # asymmetric adjacency / unsorted neighbour list / oversized query
    q = A.HostGraph.from_edges(3, [0, 0, 0], [(0, 1), (1, 2)])
    bad = q.nbrs.copy()
    bad[0], bad[1] = bad[1], bad[0]
    with pytest.raises(A.AsdmError) as e:
        A._check(A._cs_build(dg_c0._h, A._ptr(q.offsets), A._ptr(np.ascontiguousarray(q.nbrs[::-1])),
                             A._ptr(q.labels), q.n, A.C.byref(A._vp()), A.C.byref(A.C.c_int())))
    assert e.value.code == A.ERR_INVALID


def test_disconnected_query_has_no_candidates(dg_c0):
    q = A.HostGraph.from_edges(4, [0, 0, 0, 0], [(0, 1), (2, 3)])
    r = A.match(dg_c0, q)
    assert r.count == 0 and not r.nonempty


def test_batched_form_matches_golden(golden, c0_files, c0d_files, dg_c0, dg_c0d, edge_files):
    _, _, qs, _ = c0_files
    counts, status = A.run_batch(dg_c0, qs)
    assert status.tolist() == [0] * len(qs)
    assert counts.tolist() == [r["count"] for r in golden["sets"]["c0"]]
    _, _, by_size = c0d_files
    recs = golden["sets"]["c0d"]
    counts, status = A.run_batch(dg_c0d, [by_size[r["size"]][0][r["index"]] for r in recs])
    assert status.tolist() == [0] * len(recs)
    assert counts.tolist() == [r["count"] for r in recs]
    # hand-built corner cases (2-vertex query, empty candidate spaces, cliques) in one batch,
    # interleaved with ordinary queries
    recs = golden["sets"]["edge"]
    mixed = []
    for i, r in enumerate(recs):
        mixed.append(edge_files[r["name"]][0])
        mixed.append(qs[i])
    want = []
    for i, r in enumerate(recs):
        want += [r["count"], golden["sets"]["c0"][i]["count"]]
    counts, status = A.run_batch(dg_c0, mixed)
    assert status.tolist() == [0] * len(mixed)
    assert counts.tolist() == want


def test_batched_time_limit_marks_every_query(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    heavy = sorted(golden["sets"]["c0d"], key=lambda r: -r["count"])[:3]
    counts, status = A.run_batch(dg_c0d, [by_size[r["size"]][0][r["index"]] for r in heavy], time_limit_s=1e-7)
    assert all(s == A.ERR_TIMEOUT for s in status.tolist())
    counts, status = A.run_batch(dg_c0d, [by_size[r["size"]][0][r["index"]] for r in heavy])
    assert counts.tolist() == [r["count"] for r in heavy]


def test_every_tuning_gives_the_same_counts(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    recs = golden["sets"]["c0d"]
    b = A.BatchInput([by_size[r["size"]][0][r["index"]] for r in recs])
    want = [r["count"] for r in recs]
    for mb in (1, 2, 3, 4, 5, 6):
        for ll in (0, 32, 4096):
            dg_c0d.set_tuning(mb, ll)
            A.run_batch_packed(dg_c0d, b)
            assert b.counts.tolist() == want, (mb, ll)
    # intersection method: gallop only, merge up to small ratios, merge almost always
    for mr in (0, 1, 32, 1024):
        for mb in (1, 5):
            dg_c0d.set_tuning(mb, 96, merge_ratio=mr)
            A.run_batch_packed(dg_c0d, b)
            assert b.counts.tolist() == want, (mb, mr)
    dg_c0d.set_tuning(1, 96, merge_ratio=8)
    best, table = A.autotune(dg_c0d, b, reps=1, lane_leaf=(96,))
    # four kernel configurations, the other planner, two more root-block sizes, three more merge ratios
    assert len(table) == 10 and best in table
    assert {r["planner"] for r in table} == {A.PLANNER_DP, A.PLANNER_GREEDY}
    assert {r["root_block_min"] for r in table} == {16, 64, 256}
    assert {r["merge_ratio"] for r in table} == {0, 2, 8, 32}
    for rb in (1, 4, 256):
        dg_c0d.set_tuning(1, 96, A.PLANNER_DP, rb)
        A.run_batch_packed(dg_c0d, b)
        assert b.counts.tolist() == want, rb
    dg_c0d.set_tuning(1, 96, A.PLANNER_DP, 64, merge_ratio=8)


def test_batched_local_counts_match_golden_csv(golden, c0_files, c0d_files, dg_c0, dg_c0d, edge_files):
    _, _, qs, _ = c0_files
    recs = [r for r in golden["sets"]["c0"] if "csv_sha" in r]
    counts, status, mats = A.run_batch_local(dg_c0, [qs[r["index"]] for r in recs])
    assert status.tolist() == [0] * len(recs)
    for r, c, m in zip(recs, counts.tolist(), mats):
        assert c == r["count"]
        assert csv_sha(m) == r["csv_sha"], r["index"]
    _, _, by_size = c0d_files
    recs = [r for r in golden["sets"]["c0d"] if "csv_sha" in r]
    counts, status, mats = A.run_batch_local(dg_c0d, [by_size[r["size"]][0][r["index"]] for r in recs])
    for r, c, m in zip(recs, counts.tolist(), mats):
        assert c == r["count"] and csv_sha(m) == r["csv_sha"], r
    recs = [r for r in golden["sets"]["edge"] if "csv_sha" in r]
    counts, status, mats = A.run_batch_local(dg_c0, [edge_files[r["name"]][0] for r in recs])
    for r, c, m in zip(recs, counts.tolist(), mats):
        assert c == r["count"] and csv_sha(m) == r["csv_sha"], r["name"]


def test_batched_local_counts_agree_with_single_query_mode(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    recs = sorted(golden["sets"]["c0d"], key=lambda r: -r["count"])[:6]   # heaviest, beyond the golden CSVs
    qs = [by_size[r["size"]][0][r["index"]] for r in recs]
    counts, status, mats = A.run_batch_local(dg_c0d, qs)
    for r, q, c, m in zip(recs, qs, counts.tolist(), mats):
        single = A.match(dg_c0d, q, mode=A.MODE_LOCAL)
        assert c == r["count"] == single.count
        assert np.array_equal(m, single.local_counts)
        assert all(int(x) == r["count"] for x in m.sum(axis=0, dtype=np.uint64))


def test_orders_with_cartesian_vertices_give_the_golden_counts(golden, c0_files, dg_c0):
    """Orders in which a vertex has no earlier neighbour (the reference planner's
    Cartesian attributes) are accepted; the count does not depend on the order."""
    _, _, qs, _ = c0_files
    checked = 0
    for rec in golden["sets"]["c0"][:60]:
        q = qs[rec["index"]]
        adj = [set(q.nbrs[q.offsets[u]:q.offsets[u + 1]].tolist()) for u in range(q.n)]
        # start with two vertices that are not adjacent, the rest in reverse id order
        pair = next(((a, b) for a in range(q.n) for b in range(q.n) if a != b and b not in adj[a]), None)
        if pair is None:
            continue
        order = list(pair) + [u for u in reversed(range(q.n)) if u not in pair]
        assert A.match(dg_c0, q, order=order).count == rec["count"], rec["index"]
        checked += 1
    assert checked >= 30
