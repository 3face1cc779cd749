"""GPU tests of the learned-estimator path: exact prefix counts (the training
targets) against a brute-force count and the golden full counts, the
network's forward and backward passes against an fp32 numpy restatement with
the same bf16 roundings, training, and the invariant that learned plans never
change a count.  Also the staged batch API and per-query count limits."""
import numpy as np
import pytest

import asdmatch_b200 as A
from asdmatch_b200 import estimator as E

pytestmark = pytest.mark.gpu

H, IN = 128, 256
NW = H * IN


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


def _data_adjacency(g):
    off = g.offsets.astype(np.int64)
    return [set(g.nbrs[off[v]:off[v + 1]].tolist()) for v in range(g.n)]


def _brute_prefix_count(q, cand, gadj, order):
    """Injective assignments of `order`'s vertices to their candidate sets
    with every query edge among them on a data edge."""
    qadj = E.query_adjacency(q)
    pos = {u: k for k, u in enumerate(order)}
    back = [[pos[w] for w in qadj[u] if w in pos and pos[w] < k] for k, u in enumerate(order)]
    phi = [0] * len(order)

    def rec(k):
        if k == len(order):
            return 1
        u = order[k]
        if back[k]:
            js = sorted(back[k], key=lambda j: len(gadj[phi[j]]))
            opts = set(gadj[phi[js[0]]]) & cand[u]
            for j in js[1:]:
                opts &= gadj[phi[j]]
        else:
            opts = cand[u]
        used = set(phi[:k])
        total = 0
        for v in opts:
            if v in used:
                continue
            phi[k] = v
            total += rec(k + 1)
        return total

    return rec(0)


def _bfs(adj, mask, start):
    order, seen, i = [start], {start}, 0
    while i < len(order):
        for w in adj[order[i]]:
            if mask >> w & 1 and w not in seen:
                seen.add(w)
                order.append(w)
        i += 1
    return order


def test_prefix_counts_match_brute_force_and_full_counts(golden, c0_files, dg_c0):
    g, _, qs, _ = c0_files
    gadj = _data_adjacency(g)
    rng = np.random.default_rng(3)
    checked = 0
    for rec in golden["sets"]["c0"][:24]:
        q = qs[rec["index"]]
        cs = A.CandidateSpace(dg_c0, q)
        if not cs.nonempty:
            cs.close()
            continue
        cand = [set(cs.candidate_set(u).tolist()) for u in range(q.n)]
        adj = E.query_adjacency(q)
        masks = sorted(set(E.sample_subsets(q, rng, 10, kmin=2, kmax=4)) | {1 << u for u in range(2)})
        orders = [E.connected_order(adj, m) for m in masks]
        # the whole query as one prefix: its partial matches are the matches
        full = E.connected_order(adj, (1 << q.n) - 1)
        counts, status = cs.prefix_counts(orders + [full])
        assert status.tolist() == [0] * (len(orders) + 1)
        assert int(counts[-1]) == rec["count"], rec["index"]
        for o, c in zip(orders, counts[:-1].tolist()):
            assert c == _brute_prefix_count(q, cand, gadj, o), (rec["index"], o)
            checked += 1
        # a prefix's count does not depend on the order of its vertices:
        # breadth-first from the highest vertex instead of the lowest
        other = [_bfs(adj, m, m.bit_length() - 1) for m in masks]
        c2, s2 = cs.prefix_counts(other)
        assert s2.tolist() == [0] * len(other)
        assert c2.tolist() == counts[:-1].tolist()
        cs.close()
    assert checked > 100


def test_prefix_counts_reject_bad_prefixes(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    q = next(qs[r["index"]] for r in golden["sets"]["c0"] if r["cs_sha"] is not None)
    cs = A.CandidateSpace(dg_c0, q)
    adj = E.query_adjacency(q)
    bad = [[0, 0], [0, q.n + 3]]
    far = next((w for w in range(q.n) if w != 0 and w not in adj[0]), None)
    if far is not None:
        bad.append([0, far])
    counts, status = cs.prefix_counts(bad)
    assert status.tolist() == [A.ERR_INVALID] * len(bad)
    cs.close()


def _bf(a):
    return A.from_bf16_bits(A.to_bf16_bits(np.asarray(a, np.float32)))


def _segment_sum(rows, adj_off, adj, n):
    out = np.zeros((n, rows.shape[1]), np.float64)
    src = np.repeat(np.arange(n), np.diff(adj_off.astype(np.int64)))
    np.add.at(out, src, rows[adj.astype(np.int64)])
    return out


def _np_forward(p, x, adj_off, adj, gid, ng):
    W = [p[l * NW:(l + 1) * NW].reshape(H, IN) for l in range(3)]
    b = [p[3 * NW + l * H:3 * NW + (l + 1) * H] for l in range(3)]
    wo, bo = p[3 * NW + 3 * H:3 * NW + 4 * H], p[-1]
    n = x.shape[0]
    h = np.zeros((n, H), np.float64)
    h[:, :x.shape[1]] = x
    Xs, Zs, Wb = [], [], [_bf(w).astype(np.float64) for w in W]
    for l in range(3):
        s = _segment_sum(h, adj_off, adj, n)
        X = np.concatenate([_bf(h), _bf(s)], axis=1).astype(np.float64)
        Z = X @ Wb[l].T + b[l]
        Xs.append(X)
        Zs.append(Z)
        h = np.maximum(Z, 0)
    gsum = np.zeros((ng, H))
    np.add.at(gsum, gid.astype(np.int64), h)
    return gsum @ wo + bo, dict(Xs=Xs, Zs=Zs, Wb=Wb, g=gsum, wo=wo)


def _np_grad(p, x, adj_off, adj, gid, ng, t):
    y, c = _np_forward(p, x, adj_off, adj, gid, ng)
    r = y - t
    loss = float(np.mean(r * r))
    dy = 2 * r / ng
    grad = np.zeros_like(p, dtype=np.float64)
    grad[3 * NW + 3 * H:3 * NW + 4 * H] = c["g"].T @ dy
    grad[-1] = dy.sum()
    dh = dy[gid.astype(np.int64)][:, None] * c["wo"][None, :]
    n = x.shape[0]
    for l in (2, 1, 0):
        d = dh * (c["Zs"][l] > 0)
        dzb = _bf(d).astype(np.float64)
        grad[3 * NW + l * H:3 * NW + (l + 1) * H] = d.sum(0)
        grad[l * NW:(l + 1) * NW] = (dzb.T @ c["Xs"][l]).reshape(-1)
        if l:
            dX = dzb @ c["Wb"][l]
            dh = dX[:, :H] + _segment_sum(dX[:, H:], adj_off, adj, n)
    return loss, grad, y


def _feature_batch(dg, q, k=5, count=40, seed=0):
    cs = A.CandidateSpace(dg, q)
    masks = E.sample_subsets(q, np.random.default_rng(seed), count, kmin=2, kmax=k)
    x, off, adj, gid = A.subset_features(cs, masks)
    cs.close()
    return x, off, adj, gid, len(masks)


def test_subset_features_layout(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    q = next(qs[r["index"]] for r in golden["sets"]["c0"] if r["cs_sha"] is not None)
    x, off, adj, gid, ng = _feature_batch(dg_c0, q)
    assert x.shape[1] == A.EST_FEATURES
    assert np.all(np.diff(gid.astype(np.int64)) >= 0) and gid[-1] == ng - 1
    # one-hot label block, the constant feature, symmetric local adjacency inside each sub-query
    assert np.all(x[:, :32].sum(1) == 1) and np.all(x[:, 40] == 1)
    src = np.repeat(np.arange(len(gid)), np.diff(off.astype(np.int64)))
    assert np.all(gid[src] == gid[adj])
    pairs = set(zip(src.tolist(), adj.tolist()))
    assert all((b, a) in pairs for a, b in pairs)
    assert np.allclose(x[:, 33] * 8, np.diff(off.astype(np.int64)))


def test_estimator_forward_matches_numpy(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    q = next(qs[r["index"]] for r in golden["sets"]["c0"] if r["cs_sha"] is not None)
    x, off, adj, gid, ng = _feature_batch(dg_c0, q, count=60)
    est = A.Estimator(A.EST_FEATURES, seed=5)
    y = est.predict(x, off, adj, gid, ng)
    want, _ = _np_forward(est.params().astype(np.float64), x, off, adj, gid, ng)
    # same bf16 roundings; only the fp32 summation order differs
    np.testing.assert_allclose(y, want, rtol=2e-2, atol=2e-2)


def test_estimator_backward_and_adam_step_match_numpy(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    q = next(qs[r["index"]] for r in golden["sets"]["c0"] if r["cs_sha"] is not None)
    x, off, adj, gid, ng = _feature_batch(dg_c0, q, count=60, seed=1)
    t = np.random.default_rng(2).uniform(0, 8, ng).astype(np.float32)
    est = A.Estimator(A.EST_FEATURES, seed=6)
    p0 = est.params()
    loss_np, grad, _ = _np_grad(p0.astype(np.float64), x, off, adj, gid, ng, t)
    lr = 1e-3
    loss = est.train_step(x, off, adj, gid, t, lr=lr)
    assert abs(loss - loss_np) <= 1e-2 * max(1.0, loss_np)
    # first Adam step: p1 - p0 = -lr * g / (|g| + 1e-8), i.e. -lr * sign(g) where g matters
    dp = est.params() - p0
    for lo, hi in ((0, 3 * NW), (3 * NW, len(p0))):
        g = grad[lo:hi]
        big = np.abs(g) > 1e-2 * np.abs(g).max()
        agree = np.sign(dp[lo:hi][big]) == -np.sign(g[big])
        assert agree.mean() > 0.98, (lo, agree.mean())
        assert np.allclose(np.abs(dp[lo:hi][big]), lr, rtol=1e-2)


def test_estimator_training_fits_prefix_counts(dg_c0, c0_files):
    g = c0_files[0]
    qs = [g.random_walk_query(8, 7000 + i, 0) for i in range(60)]
    ds = E.collect(dg_c0, qs[:48], np.random.default_rng(0), per_query=16)
    hs = E.collect(dg_c0, qs[48:], np.random.default_rng(1), per_query=16)
    assert len(ds) > 300 and len(hs) > 50
    est = A.Estimator(A.EST_FEATURES, seed=3)
    losses = E.train(est, ds, epochs=30, batch=128, lr=2e-3)
    assert losses[-1] < 0.2 * losses[0]
    ev = E.evaluate(est, hs)
    assert ev["learned"]["p50"] < 4.0
    # params round-trip
    est2 = A.Estimator(A.EST_FEATURES, seed=9)
    est2.set_params(est.params())
    x, off, adj, gid, _ = ds.batch(list(range(32)))
    np.testing.assert_array_equal(est.predict(x, off, adj, gid, 32), est2.predict(x, off, adj, gid, 32))


def test_learned_plans_never_change_counts(golden, c0_files, c0d_files, dg_c0, dg_c0d, edge_files):
    est = A.Estimator(A.EST_FEATURES, seed=11)
    _, _, by_size = c0d_files
    recs = golden["sets"]["c0d"]
    qs = [by_size[r["size"]][0][r["index"]] for r in recs]
    b = A.BatchInput(qs)
    A.run_batch_ex(dg_c0d, b, estimator=est)
    assert b.status.tolist() == [0] * len(qs)
    assert b.counts.tolist() == [r["count"] for r in recs]
    for kmax in (3, 4, 8):
        b = A.BatchInput(qs)
        A.run_batch_ex(dg_c0d, b, estimator=est, learned_max_subset=kmax)
        assert b.counts.tolist() == [r["count"] for r in recs]
    # staged form: candidate spaces, learned plans, one planned launch
    css = A.candidate_spaces(dg_c0d, qs)
    plans = A.plans_learned(css, est)
    counts, status, st = A.run_planned(css, plans)
    assert status.tolist() == [0] * len(qs)
    assert counts.tolist() == [r["count"] for r in recs]
    assert st.count == sum(r["count"] for r in recs)
    for p, q in zip(plans, qs):
        assert sorted(p.order()) == list(range(q.n))
    # corner cases (empty candidate spaces, 2-vertex and clique queries) through the learned planner
    erecs = golden["sets"]["edge"]
    b = A.BatchInput([edge_files[r["name"]][0] for r in erecs])
    A.run_batch_ex(dg_c0, b, estimator=est)
    assert b.status.tolist() == [0] * len(erecs)
    assert b.counts.tolist() == [r["count"] for r in erecs]


def test_candidate_space_batch_equals_single_builds(golden, c0_files, dg_c0):
    _, _, qs, _ = c0_files
    recs = golden["sets"]["c0"][:40]
    css = A.candidate_spaces(dg_c0, [qs[r["index"]] for r in recs])
    for r, cs in zip(recs, css):
        assert cs is not None
        assert cs.nonempty == (r["cs_sha"] is not None)
        if cs.nonempty:
            import hashlib
            assert hashlib.sha256(cs.write_to_stream().encode()).hexdigest() == r["cs_sha"], r["index"]
        cs.close()


def test_batch_count_limit_statuses(golden, c0d_files, dg_c0d):
    _, _, by_size = c0d_files
    recs = golden["sets"]["c0d"]
    qs = [by_size[r["size"]][0][r["index"]] for r in recs]
    limit = int(np.median([r["count"] for r in recs]))
    b = A.BatchInput(qs)
    A.run_batch_ex(dg_c0d, b, count_limit=limit)
    for r, c, s in zip(recs, b.counts.tolist(), b.status.tolist()):
        if r["count"] > limit:
            assert s == A.ERR_LIMIT, r
        else:
            assert s == 0 and c == r["count"], r
    # plan caches: a card for every query changes no count
    cards = []
    for q in qs:
        cs = A.CandidateSpace(dg_c0d, q)
        c = A.Card()
        for u, n in enumerate(cs.sizes().tolist()):
            c[1 << u] = float(n)
        cards.append(c)
        cs.close()
    b = A.BatchInput(qs)
    A.run_batch_ex(dg_c0d, b, cards=cards)
    assert b.counts.tolist() == [r["count"] for r in recs]


def test_both_planners_give_the_golden_counts(golden, c0_files, c0d_files, dg_c0, dg_c0d, edge_files):
    _, _, qs0, _ = c0_files
    _, _, by_size = c0d_files
    recs = golden["sets"]["c0d"]
    qs = [by_size[r["size"]][0][r["index"]] for r in recs]
    try:
        for planner in (A.PLANNER_DP, A.PLANNER_GREEDY):
            dg_c0d.set_tuning(1, 96, planner)
            dg_c0.set_tuning(1, 96, planner)
            assert dg_c0d.tuning()["planner"] == planner
            counts, status = A.run_batch(dg_c0d, qs)
            assert status.tolist() == [0] * len(qs)
            assert counts.tolist() == [r["count"] for r in recs]
            for r, q in list(zip(recs, qs))[::8]:
                cs = A.CandidateSpace(dg_c0d, q)
                p = A.Plan(cs)
                o = p.order()
                adj = E.query_adjacency(q)
                assert sorted(o) == list(range(q.n))
                assert all(any(w in adj[o[k]] for w in o[:k]) for k in range(1, q.n))
                assert A.adaptive_share_join(cs, p).count == r["count"]
                cs.close()
            erecs = golden["sets"]["edge"]
            counts, status = A.run_batch(dg_c0, [edge_files[r["name"]][0] for r in erecs])
            assert counts.tolist() == [r["count"] for r in erecs]
            counts, status = A.run_batch(dg_c0, qs0[:60])
            assert counts.tolist() == [r["count"] for r in golden["sets"]["c0"][:60]]
    finally:
        dg_c0d.set_tuning(1, 96, A.PLANNER_DP)
        dg_c0.set_tuning(1, 96, A.PLANNER_DP)
    with pytest.raises(A.AsdmError):
        dg_c0.set_tuning(1, 96, 7)
