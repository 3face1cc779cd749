"""GPU tests of the sampling estimator (asdm_card_sample), the device
counterpart of the reference's cardEstimateLabeled (plan/estimator.cpp:173-291):
its estimates of sub-query cardinalities against exact partial-match counts,
and plans made from them against the golden counts (plans never change a
count)."""
import numpy as np
import pytest

import asdmatch_b200 as A
from asdmatch_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _connected_order(q, mask):
    adj = [set(q.nbrs[q.offsets[u]:q.offsets[u + 1]].tolist()) for u in range(q.n)]
    verts = [u for u in range(q.n) if mask >> u & 1]
    order = [verts[0]]
    while len(order) < len(verts):
        nxt = next(u for u in verts if u not in order and adj[u] & set(order))
        order.append(nxt)
    return order


def _subsets(q, size):
    adj = [set(q.nbrs[q.offsets[u]:q.offsets[u + 1]].tolist()) for u in range(q.n)]
    out = set()
    for u in range(q.n):
        frontier = {1 << u}
        for _ in range(size - 1):
            frontier = {S | (1 << w) for S in frontier for v in range(q.n) if S >> v & 1 for w in adj[v]
                        if not S >> w & 1}
        out |= frontier
    return sorted(out)


def test_sampled_cardinalities_track_exact_partial_match_counts(c0d_files):
    g, _, by_size = c0d_files
    dg = A.DeviceGraph(g)
    qerr = []
    for q in by_size[8][0][:12]:
        cs = A.CandidateSpace(dg, q)
        if not cs.nonempty:
            cs.close()
            continue
        card = A.Card.sample(cs, max_subset=4, walks=4096, seed=7)
        masks = _subsets(q, 3) + _subsets(q, 4)
        exact, status = cs.prefix_counts([_connected_order(q, m) for m in masks])
        for m, c, st in zip(masks, exact.tolist(), status.tolist()):
            assert st == A.OK
            est = card[m]
            if c == 0:
                assert est == 0.0  # no walk can reach an empty level
                continue
            qerr.append(max(est / c, c / est) if est > 0 else float("inf"))
        cs.close()
    dg.close()
    qerr.sort()
    assert len(qerr) >= 100
    assert qerr[len(qerr) // 2] <= 1.2, qerr[len(qerr) // 2]
    assert qerr[int(0.9 * len(qerr))] <= 2.0, qerr[int(0.9 * len(qerr))]


def test_plans_from_sampled_cardinalities_give_the_golden_counts(golden, c0_files):
    g, _, qs, _ = c0_files
    dg = A.DeviceGraph(g)
    for rec in golden["sets"]["c0"][:40]:
        cs = A.CandidateSpace(dg, qs[rec["index"]])
        if cs.nonempty:
            card = A.Card.sample(cs, walks=256, seed=1)
            assert card.info()["entries"] > 0
            assert A.adaptive_share_join(cs, A.Plan(cs, card=card)).count == rec["count"]
        cs.close()
    dg.close()
