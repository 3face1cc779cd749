"""Seeded synthetic workloads (shapes of the reference benchmark configs),
generated with the product's own generators so every machine rebuilds the
same graphs and queries from the seeds."""
from __future__ import annotations

import os

import asdmatch_b200 as A

# config 0: N=3,112, M=12,519, exponent 2.5, 71 labels Zipf(1.0), 8-vertex queries
C0 = dict(n=3112, m=12519, gamma=2.5, nlabels=71, zipf_s=1.0, seed=1)
C0_QUERY_SEED = 1000
# a denser cousin of config 0 (fewer labels) whose queries have many matches
C0D = dict(n=3112, m=12519, gamma=2.5, nlabels=8, zipf_s=1.0, seed=2)
C0D_QUERY_SEED = 3000


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
