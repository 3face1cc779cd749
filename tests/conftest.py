import json
import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(HERE, "golden", "golden.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def workdir(tmp_path_factory):
    return str(tmp_path_factory.mktemp("asdm"))


@pytest.fixture(scope="session")
def c0_files(workdir):
    """config-0 graph and its golden queries written as t/v/e files."""
    from asdmatch_b200 import workloads as W
    g = W.graph(W.C0)
    d = os.path.join(workdir, "c0")
    dpath, _ = W.write_workload(d, g, [])
    qs = W.queries(g, 8, 200, W.C0_QUERY_SEED + 800)
    _, qpaths = W.write_workload(d, g, qs, prefix="s8_")
    return g, dpath, qs, qpaths


@pytest.fixture(scope="session")
def c0d_files(workdir):
    from asdmatch_b200 import workloads as W
    g = W.graph(W.C0D)
    d = os.path.join(workdir, "c0d")
    dpath, _ = W.write_workload(d, g, [])
    out = {}
    for size in (6, 8):
        qs = W.queries(g, size, 40, W.C0D_QUERY_SEED + 100 * size)
        _, qpaths = W.write_workload(d, g, qs, prefix="s%d_" % size)
        out[size] = (qs, qpaths)
    return g, dpath, out


@pytest.fixture(scope="session")
def edge_files(workdir, c0_files):
    import asdmatch_b200 as A
    from golden.make_golden import edge_case_queries
    d = os.path.join(workdir, "edge")
    os.makedirs(d, exist_ok=True)
    out = {}
    for name, n, labels, edges in edge_case_queries():
        q = A.HostGraph.from_edges(n, labels, edges)
        p = os.path.join(d, name + ".graph")
        q.write(p)
        out[name] = (q, p)
    return out


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
