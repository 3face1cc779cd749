"""Workload specifications (graph parameters, query seeds and sizes) as plain
data, with no dependency on the compiled library: a process that only writes
input files for another implementation (bench.py's reference arm) loads this
file by path and runs the host-only generator asdmatch_b200/bin/asdm_gen.out.

* C0  — N=3,112, M=12,519, degree exponent 2.5, 71 labels Zipf(1.0), 8-vertex
        random-walk queries (the shape of the Yeast benchmark).
* C0D — the same graph shape with 8 labels (heavier enumeration for tests).
* C1  — N=3.77M, M=16.5M, exponent 2.1, 20 labels Zipf(1.2) (the shape of US
        Patents), resident in HBM.
* C2  — the C1 graph with the mixed batch: query i has seed C2_QUERY_SEED + i
        and a size uniform in 4..32 (c2_size).
* C1 queries — 100 queries each of 12 and 16 vertices on the C1 graph, half
        dense (average query degree >= 3) and half sparse (< 3): c1_seed_base.
* C4  — local subgraph counting: N=1.0M, M=10M, exponent 2.3, 32 labels
        Zipf(1.0), 50 random-walk queries of 10 vertices: c4_query_specs.
"""

C0 = dict(n=3112, m=12519, gamma=2.5, nlabels=71, zipf_s=1.0, seed=1)
C0_QUERY_SEED = 1000
C0D = dict(n=3112, m=12519, gamma=2.5, nlabels=8, zipf_s=1.0, seed=2)
C0D_QUERY_SEED = 3000
C1 = dict(n=3_770_000, m=16_500_000, gamma=2.1, nlabels=20, zipf_s=1.2, seed=11)
C2_QUERY_SEED = 50_000
C2_QUERIES = 1000
C1_QUERY_SEED = 70_000
C4 = dict(n=1_000_000, m=10_000_000, gamma=2.3, nlabels=32, zipf_s=1.0, seed=41)
C4_QUERY_SEED = 90_000
C4_QUERIES = 50
C4_QUERY_SIZE = 10
DENSE, SPARSE = 1, 2  # density argument of the query generator


def c2_seed_size(i):
    """(seed, size) of the i-th query of the C2 mixed batch: sizes uniform in
    4..32, decorrelated from the walk seed."""
    seed = C2_QUERY_SEED + i
    return seed, 4 + (seed * 2654435761 % 2 ** 32) % 29


def c1_seed_base(size, density):
    """First walk seed tried for the config-1 queries of one size and density;
    the queries are the first 50 seeds from there whose walk yields a query of
    that density (a dense walk is not found from every seed)."""
    return C1_QUERY_SEED + 10_000 * size + 1_000 * density


C1_SIZES = (12, 16)
C1_PER_CLASS = 50


def c4_query_specs():
    """(size, seed, density) of the config-4 queries."""
    return [(C4_QUERY_SIZE, C4_QUERY_SEED + i, 0) for i in range(C4_QUERIES)]


C4_PARITY_SEED = 95_000
C4_PARITY = 40
C4_EMBED_SEED = 96_000


def c4_parity_specs():
    """(size, seed, density) of the config-4 parity queries: random-walk
    queries of 4..8 vertices on the config-4 graph, small enough for the
    reference's local counting to finish, so that its |Vg| x |Vq| CSV can be
    compared at the graph's full size."""
    return [(4 + i % 5, C4_PARITY_SEED + i, 0) for i in range(C4_PARITY)]


def generator_args(spec):
    """The graph arguments of asdm_gen.out for a spec."""
    return [str(spec["n"]), str(spec["m"]), repr(float(spec["gamma"])), str(spec["nlabels"]),
            repr(float(spec["zipf_s"])), str(spec["seed"])]
