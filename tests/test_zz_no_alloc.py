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


def _noalloc_rc(cs, plan, count_limit=0):
    st = A.RunStats()
    rc = _noalloc(cs._h, plan._h, 0.0, count_limit, C.byref(st))
    return rc, st


def _count_noalloc(cs, plan):
    rc, st = _noalloc_rc(cs, plan)
    A._check(rc, "noalloc")
    return st.count


class _PoolWatch:
    """High-water mark of the device's default stream-ordered pool, which the
    library's other entry points allocate from (cudaMallocAsync)."""

    def __init__(self, device=0):
        from cuda.bindings import driver, runtime as rt
        self.rt = rt
        self.u64 = driver.cuuint64_t
        err, self.pool = rt.cudaDeviceGetDefaultMemPool(device)
        assert err == rt.cudaError_t.cudaSuccess

    def _attr(self, a):
        err, v = self.rt.cudaMemPoolGetAttribute(self.pool, a)
        assert err == self.rt.cudaError_t.cudaSuccess
        return int(v)

    def reset(self):
        rt = self.rt
        (err,) = rt.cudaMemPoolSetAttribute(self.pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh,
                                            self.u64(0))
        assert err == rt.cudaError_t.cudaSuccess
        return self._attr(rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)

    def high(self):
        return self._attr(self.rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)


def test_noalloc_count_matches_run_plan_twice_in_a_row():
    g = W.graph(W.C0D)
    dg = A.DeviceGraph(g)
    qs = W.queries(g, 8, 6, W.C0D_QUERY_SEED + 800) + W.queries(g, 6, 4, W.C0D_QUERY_SEED + 600)
    watch = _PoolWatch()
    checked = 0
    for q in qs:
        cs = A.CandidateSpace(dg, q)
        if not cs.nonempty:
            cs.close()
            continue
        plan = A.Plan(cs)
        want = A.adaptive_share_join(cs, plan).count
        # two calls in a row: the shared scratch keeps the previous call's contents;
        # neither call takes memory from the pool the library otherwise uses
        used = watch.reset()
        assert _count_noalloc(cs, plan) == want
        assert _count_noalloc(cs, plan) == want
        assert watch.high() == used
        if checked == 0:
            # the watch sees the allocating entry point's scratch
            used = watch.reset()
            A.adaptive_share_join(cs, plan)
            assert watch.high() > used
        if want > 1 and checked < 3:
            # the count limit stops the run with ASDM_ERR_LIMIT; the next call is unaffected
            rc, st = _noalloc_rc(cs, plan, count_limit=1)
            assert rc == A.ERR_LIMIT and st.count >= 1
            assert _count_noalloc(cs, plan) == want
        cs.close()
        checked += 1
    assert checked >= 5
    dg.close()
