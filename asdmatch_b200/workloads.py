"""Seeded synthetic workloads with the shapes of the reference benchmark
configurations, built with the library's own generators so that every
machine rebuilds identical graphs and queries from the seeds.

* C0  — N=3,112, M=12,519, degree exponent 2.5, 71 labels Zipf(1.0), 8-vertex
        random-walk queries (the shape of the Yeast benchmark).
* C0D — the same graph shape with 8 labels, whose queries have 10^3..10^8
        matches (heavier enumeration for parity tests).
* C1  — N=3.77M, M=16.5M, exponent 2.1, 20 labels Zipf(1.2) (the shape of US
        Patents), resident in HBM.
* C2  — the C1 graph with a mixed batch of random-walk queries whose sizes are
        uniform in 4..32.  ``screen`` keeps the first queries (in seed order)
        whose exact match count is at most ``count_limit``; the kept seeds and
        counts are stored in ``c2_screened.json`` beside this module.
* C4  — local subgraph counting: N=1.0M, M=10M, exponent 2.3, 32 labels
        Zipf(1.0).  No 10-vertex random-walk query of 1,500 tried has <= 10^9
        matches, so ``screen_c4`` keeps 8-vertex ones (``c4_screened.json``).
"""
from __future__ import annotations

import json
import os

import asdmatch_b200 as A

C0 = dict(n=3112, m=12519, gamma=2.5, nlabels=71, zipf_s=1.0, seed=1)
C0_QUERY_SEED = 1000
C0D = dict(n=3112, m=12519, gamma=2.5, nlabels=8, zipf_s=1.0, seed=2)
C0D_QUERY_SEED = 3000
C1 = dict(n=3_770_000, m=16_500_000, gamma=2.1, nlabels=20, zipf_s=1.2, seed=11)
C2_QUERY_SEED = 50_000
C2_COUNT_LIMIT = 10 ** 9
C2_SCREEN_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_screened.json")
# config 4: local subgraph counting; N=1.0M, M=10M, exponent 2.3, 32 labels Zipf(1.0), 10-vertex queries
C4 = dict(n=1_000_000, m=10_000_000, gamma=2.3, nlabels=32, zipf_s=1.0, seed=41)
C4_QUERY_SEED = 90_000
C4_SCREEN_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c4_screened.json")


def graph(spec):
    return A.HostGraph.chung_lu(spec["n"], spec["m"], spec["gamma"], spec["nlabels"], spec["zipf_s"], spec["seed"])


def queries(g, size, count, seed0, density=0):
    return [g.random_walk_query(size, seed0 + i, density) for i in range(count)]


def write_workload(dirpath, g, qs, prefix="q"):
    os.makedirs(dirpath, exist_ok=True)
    dpath = os.path.join(dirpath, "data.graph")
    if not os.path.exists(dpath):
        g.write(dpath)
    qpaths = []
    for i, q in enumerate(qs):
        p = os.path.join(dirpath, "%s%d.graph" % (prefix, i))
        q.write(p)
        qpaths.append(p)
    return dpath, qpaths


def c2_candidate(g, i):
    """The i-th candidate query of the C2 mixed batch: (seed, size, query)."""
    seed = C2_QUERY_SEED + i
    size = 4 + (seed * 2654435761 % 2 ** 32) % 29  # uniform in 4..32, decorrelated from the walk seed
    return seed, size, g.random_walk_query(size, seed, 0)


def screen(dg, g, keep=1000, count_limit=C2_COUNT_LIMIT, time_limit_s=5.0, max_candidates=20000, log=None):
    """Exact counts of C2 candidates in seed order; keeps those <= count_limit."""
    kept, rejected = [], 0
    for i in range(max_candidates):
        if len(kept) >= keep:
            break
        seed, size, q = c2_candidate(g, i)
        try:
            r = A.count_query(dg, q, time_limit_s=time_limit_s, count_limit=count_limit)
            kept.append(dict(index=i, seed=seed, size=size, edges=q.m2 // 2, count=r.count))
        except A.AsdmError as e:
            if e.code not in (A.ERR_LIMIT, A.ERR_TIMEOUT, A.ERR_OVERFLOW):
                raise
            rejected += 1
        if log and (i + 1) % 100 == 0:
            log("screened %d kept %d" % (i + 1, len(kept)))
    return dict(spec=C1, query_seed=C2_QUERY_SEED, count_limit=count_limit, time_limit_s=time_limit_s,
                candidates=len(kept) + rejected, rejected=rejected, queries=kept)


def c4_candidate(g, i, size=10):
    """The i-th candidate query of the config-4 set: (seed, size, query)."""
    seed = C4_QUERY_SEED + i
    return seed, size, g.random_walk_query(size, seed, 0)


def screen_c4(dg, g, keep=50, size=8, count_limit=C2_COUNT_LIMIT, time_limit_s=2.0, max_candidates=4000, log=None):
    """Config-4 queries in seed order whose exact count is <= count_limit."""
    kept, rejected = [], 0
    for i in range(max_candidates):
        if len(kept) >= keep:
            break
        seed, sz, q = c4_candidate(g, i, size)
        try:
            r = A.count_query(dg, q, time_limit_s=time_limit_s, count_limit=count_limit)
            kept.append(dict(index=i, seed=seed, size=sz, edges=q.m2 // 2, count=r.count))
        except A.AsdmError as e:
            if e.code not in (A.ERR_LIMIT, A.ERR_TIMEOUT, A.ERR_OVERFLOW):
                raise
            rejected += 1
        if log and (i + 1) % 250 == 0:
            log("c4 screened %d kept %d" % (i + 1, len(kept)))
    return dict(spec=C4, query_seed=C4_QUERY_SEED, size=size, count_limit=count_limit, time_limit_s=time_limit_s,
                candidates=len(kept) + rejected, rejected=rejected, queries=kept)


def load_c4_screen():
    with open(C4_SCREEN_FILE) as fh:
        return json.load(fh)


def c4_queries(g, screen_data):
    out = []
    for rec in screen_data["queries"]:
        seed, size, q = c4_candidate(g, rec["index"], screen_data["size"])
        assert seed == rec["seed"]
        out.append(q)
    return out


def load_c2_screen():
    with open(C2_SCREEN_FILE) as fh:
        return json.load(fh)


def c2_queries(g, screen_data):
    """Regenerates the screened C2 queries from their indices."""
    out = []
    for rec in screen_data["queries"]:
        seed, size, q = c2_candidate(g, rec["index"])
        assert seed == rec["seed"] and size == rec["size"]
        out.append(q)
    return out


if __name__ == "__main__":
    # python -m asdmatch_b200.workloads c2 [keep] [out]   |   ... c4 [keep] [out] [size]
    import sys
    import time
    t = time.time()
    which = sys.argv[1] if len(sys.argv) > 1 else "c2"
    keep = int(sys.argv[2]) if len(sys.argv) > 2 else (1000 if which == "c2" else 50)
    if which == "c2":
        g = graph(C1)
        dg = A.DeviceGraph(g)
        data = screen(dg, g, keep=keep, log=print)
        out = sys.argv[3] if len(sys.argv) > 3 else C2_SCREEN_FILE
    else:
        g = graph(C4)
        dg = A.DeviceGraph(g)
        size = int(sys.argv[4]) if len(sys.argv) > 4 else 8
        data = screen_c4(dg, g, keep=keep, size=size, log=print)
        out = sys.argv[3] if len(sys.argv) > 3 else C4_SCREEN_FILE
    with open(out, "w") as fh:
        json.dump(data, fh, indent=0)
    print("screen done in %.1f s: kept %d of %d" % (time.time() - t, len(data["queries"]), data["candidates"]))
