"""The allocation-free counting entry point (asdm_run_plan_count_noalloc).

Callers whose device memory is fully reserved by their own pool, or that
cannot take cudaMalloc/cudaFree (and the synchronisation they imply) in the
middle of their work, count through this entry point: its scratch is a fixed
file-scope device array instead of library allocations.  This file is
collected last, so a failure here leaves every other test already run.
"""
import ctypes as C

import pytest

import asdmatch_b200 as A
from asdmatch_b200 import workloads as W

pytestmark = pytest.mark.gpu

_noalloc = A._lib.asdm_run_plan_count_noalloc
_noalloc.restype = C.c_int
_noalloc.argtypes = [A._vp, A._vp, C.c_double, C.c_uint64, C.POINTER(A.RunStats)]


def _count_noalloc(cs, plan):
    st = A.RunStats()
    A._check(_noalloc(cs._h, plan._h, 0.0, 0, C.byref(st)), "noalloc")
    return st.count


def test_noalloc_count_matches_run_plan_twice_in_a_row():
    g = W.graph(W.C0D)
    dg = A.DeviceGraph(g)
    qs = W.queries(g, 8, 6, W.C0D_QUERY_SEED + 800) + W.queries(g, 6, 4, W.C0D_QUERY_SEED + 600)
    checked = 0
    for q in qs:
        cs = A.CandidateSpace(dg, q)
        if not cs.nonempty:
            cs.close()
            continue
        plan = A.Plan(cs)
        want = A.adaptive_share_join(cs, plan).count
        # two calls in a row: the shared scratch keeps the previous call's contents
        assert _count_noalloc(cs, plan) == want
        assert _count_noalloc(cs, plan) == want
        cs.close()
        checked += 1
    assert checked >= 5
    dg.close()
