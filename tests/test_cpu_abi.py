"""CPU-only checks of the C-ABI library: it loads, exports every declared
entry point, and its host-side logic (loader, writer, generators, argument
validation) behaves like the reference's loader."""
import os
import re

import numpy as np
import pytest

import asdmatch_b200 as A
import oracle_util as O
from asdmatch_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "asdm.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(asdm_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 24
    for n in names:
        assert hasattr(A._lib, n), n


def test_version_string():
    assert "sm_100a" in A.version()


def test_missing_file_is_io_error(tmp_path):
    with pytest.raises(A.AsdmError) as e:
        A.load_graph_from_text_file(str(tmp_path / "nope.graph"))
    assert e.value.code == A.ERR_IO
    assert "Can not open file" in str(e.value)


def test_loader_layout_and_round_trip(tmp_path):
    # the README sample graph (t/v/e), with a trailing edge-label token like the yeast queries
    p = tmp_path / "s.graph"
    p.write_text("t 5 6\nv 0 0 2\nv 1 1 3\nv 2 2 3\nv 3 1 2\nv 4 2 2\n"
                 "e 0 1 0\ne 0 2 0\ne 1 2 0\ne 1 3 0\ne 2 4 0\ne 3 4 0\n")
    g = A.load_graph_from_text_file(str(p))
    assert (g.n, g.m2, g.nlabels) == (5, 12, 3)
    for v in range(g.n):
        nb = g.nbrs[g.offsets[v]:g.offsets[v + 1]].tolist()
        assert nb == sorted(nb, key=lambda x: (g.labels[x], x))
    assert g.nbrs[g.offsets[1]:g.offsets[2]].tolist() == [0, 3, 2]   # labels 0,1,2
    q = tmp_path / "w.graph"
    g.write(str(q))
    g2 = A.load_graph_from_text_file(str(q))
    assert np.array_equal(g.offsets, g2.offsets) and np.array_equal(g.nbrs, g2.nbrs)
    assert np.array_equal(g.labels, g2.labels)


@pytest.mark.parametrize("text", [
    "t 2 1\nv 0 0 1\nv 1 0 2\ne 0 1\n",          # declared degree does not match
    "t 2 1\nv 0 0 1\nv 1 0 1\ne 0 5\n",          # endpoint out of range
    "t 2 1\nv 1 0 1\nv 0 0 1\ne 0 1\n",          # vertex lines out of order
])
def test_loader_rejects_malformed(tmp_path, text):
    p = tmp_path / "bad.graph"
    p.write_text(text)
    with pytest.raises(A.AsdmError) as e:
        A.load_graph_from_text_file(str(p))
    assert e.value.code == A.ERR_INVALID


def test_from_edges_rejects_loops_and_duplicates():
    with pytest.raises(A.AsdmError):
        A.HostGraph.from_edges(3, [0, 0, 0], [(0, 0)])
    with pytest.raises(A.AsdmError):
        A.HostGraph.from_edges(3, [0, 0, 0], [(0, 1), (1, 0)])


def test_generator_is_pinned_by_golden_digests(golden, tmp_path):
    for name, spec in (("c0", W.C0), ("c0d", W.C0D)):
        g = W.graph(spec)
        p = tmp_path / (name + ".graph")
        g.write(str(p))
        assert O.sha256_file(str(p)) == golden["generator"][name]["data_sha"]
        assert g.m2 == 2 * spec["m"]


def test_chung_lu_shape():
    g = W.graph(W.C0)
    deg = np.diff(g.offsets.astype(np.int64))
    assert g.n == 3112 and g.m2 == 2 * 12519
    # structural cutoff: the largest expected degree is sqrt(2M)
    assert deg.max() < 4 * np.sqrt(2 * 12519)
    hist = np.bincount(g.labels, minlength=71)
    assert hist[0] > hist[10] > 0   # Zipf-ordered labels


def test_random_walk_queries_are_connected_induced_subgraphs():
    g = W.graph(W.C0D)
    for seed in range(20):
        for density in (0, 1, 2):
            try:
                q = g.random_walk_query(8, seed, density)
            except A.AsdmError:
                continue
            assert q.n == 8
            seen, stack = {0}, [0]
            while stack:
                u = stack.pop()
                for w in q.nbrs[q.offsets[u]:q.offsets[u + 1]]:
                    if int(w) not in seen:
                        seen.add(int(w))
                        stack.append(int(w))
            assert len(seen) == 8
            avg = q.m2 / q.n
            if density == 1:
                assert avg >= 3
            if density == 2:
                assert avg < 3


@pytest.mark.skipif(__import__("conftest").cuda_available(), reason="checks the no-GPU error path")
def test_device_entry_points_fail_cleanly_without_gpu():
    g = W.graph(W.C0)
    with pytest.raises(A.AsdmError) as e:
        A.DeviceGraph(g)
    assert e.value.code == A.ERR_CUDA


def test_graph_close_frees_its_candidate_spaces_first():
    """A candidate space frees its device memory on its graph's stream, so
    DeviceGraph.close() closes the candidate spaces still alive on it before
    freeing the graph (host bookkeeping only: stand-in handles, no device)."""
    import weakref

    class StandInGraph:
        pass

    g = StandInGraph()
    g._spaces = weakref.WeakSet()
    g._h = None
    spaces = [A.CandidateSpace._wrap(0, None, g, False) for _ in range(3)]
    assert len(g._spaces) == 3
    A.DeviceGraph.close(g)
    assert all(cs._h is None for cs in spaces)
    del spaces
    assert len(g._spaces) == 0
