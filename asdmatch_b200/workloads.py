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
* C1 queries — 100 each of 12 and 16 vertices, half dense, half sparse
        (``c1_batch``).
* C4  — local subgraph counting: N=1.0M, M=10M, exponent 2.3, 32 labels
        Zipf(1.0), 50 random-walk queries of 10 vertices (``c4_batch``).
"""
from __future__ import annotations

import json
import os

import asdmatch_b200 as A

from asdmatch_b200.specs import (C0, C0_QUERY_SEED, C0D, C0D_QUERY_SEED, C1, C1_PER_CLASS, C1_SIZES,  # noqa: F401
                                  C2_QUERIES, C2_QUERY_SEED, C4, C4_QUERY_SEED, DENSE, SPARSE, c1_seed_base,
                                  c2_seed_size, c4_parity_specs, c4_query_specs)



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
    """The config-1 queries: 100 each of 12 and 16 vertices, half dense, half
    sparse, as (size, density, seed, query) in that order."""
    out = []
    for size in C1_SIZES:
        for density in (DENSE, SPARSE):
            seed = c1_seed_base(size, density)
            found = 0
            while found < C1_PER_CLASS:
                try:
                    q = g.random_walk_query(size, seed, density)
                    out.append((size, density, seed, q))
                    found += 1
                except A.AsdmError as e:
                    if e.code != A.ERR_INVALID:
                        raise
                seed += 1
    return out


def c4_batch(g):
    """The config-4 queries: 50 random-walk queries of 10 vertices."""
    return from_specs(g, c4_query_specs())
