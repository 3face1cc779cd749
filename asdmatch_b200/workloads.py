"""Seeded synthetic workloads with the shapes of the reference benchmark
configurations, built with the library's own generators so that every
machine rebuilds identical graphs and queries from the seeds.

* C0  — N=3,112, M=12,519, degree exponent 2.5, 71 labels Zipf(1.0), 8-vertex
        random-walk queries (the shape of the Yeast benchmark).
* C0D — the same graph shape with 8 labels, whose queries have 10^3..10^8
        matches (heavier enumeration for parity tests).
* C1  — N=3.77M, M=16.5M, exponent 2.1, 20 labels Zipf(1.2) (the shape of US
        Patents), resident in HBM.
* C2  — the C1 graph with the mixed batch: the first 1,000 random-walk queries
        in seed order, sizes uniform in 4..32 (``c2_batch``), none screened out.
* C4  — local subgraph counting: N=1.0M, M=10M, exponent 2.3, 32 labels
        Zipf(1.0).  No 10-vertex random-walk query of 1,500 tried has <= 10^9
        matches, so ``screen_c4`` keeps 8-vertex ones (``c4_screened.json``).
"""
from __future__ import annotations

import json
import os

import asdmatch_b200 as A

from asdmatch_b200.specs import (C0, C0_QUERY_SEED, C0D, C0D_QUERY_SEED, C1, C2_QUERIES, C2_QUERY_SEED, C4,  # noqa: F401
                                  C4_QUERY_SEED, c1_query_specs, c2_seed_size, c4_query_specs)

C2_COUNT_LIMIT = 10 ** 9
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
    """The i-th query of the C2 mixed batch: (seed, size, query)."""
    seed, size = c2_seed_size(i)
    return seed, size, g.random_walk_query(size, seed, 0)


def c2_batch(g, count=C2_QUERIES):
    """The C2 mixed batch as specified: the first `count` queries in seed order,
    sizes uniform in 4..32, none screened out."""
    return [c2_candidate(g, i)[2] for i in range(count)]


def from_specs(g, specs):
    """Queries of (size, seed, density) specs."""
    return [g.random_walk_query(size, seed, density) for size, seed, density in specs]


def c1_batch(g):
    """The config-1 queries: 100 each of 12 and 16 vertices, half dense, half sparse."""
    return from_specs(g, c1_query_specs())


def c4_batch(g):
    """The config-4 queries: 50 random-walk queries of 10 vertices."""
    return from_specs(g, c4_query_specs())


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


if __name__ == "__main__":
    # python -m asdmatch_b200.workloads c4 [keep] [out] [size]: the config-4 local-counting screen
    import sys
    import time
    t = time.time()
    keep = int(sys.argv[2]) if len(sys.argv) > 2 else 50
    g = graph(C4)
    dg = A.DeviceGraph(g)
    size = int(sys.argv[4]) if len(sys.argv) > 4 else 8
    data = screen_c4(dg, g, keep=keep, size=size, log=print)
    out = sys.argv[3] if len(sys.argv) > 3 else C4_SCREEN_FILE
    with open(out, "w") as fh:
        json.dump(data, fh, indent=0)
    print("screen done in %.1f s: kept %d of %d" % (time.time() - t, len(data["queries"]), data["candidates"]))
