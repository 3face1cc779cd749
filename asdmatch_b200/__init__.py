"""ASDMatch-B200: the matching and counting path of ASDMatch on the B200.

A thin ctypes binding over ``libasdm_b200.so`` (C ABI in ``include/asdm.h``).
Names follow the reference's own interface so code written against it reads
the same:

* :func:`load_graph_from_text_file`  — ``Graph::loadGraphFromTextFile`` (relation/graph.cpp:68-148)
* :class:`CandidateSpace`            — ``CandidateSpace`` + ``buildCandCFL`` (relation/candidate_space.cpp)
* :func:`leapfrog_join`              — ``ComputeSetIntersection::LeapfrogJoin`` (utility/compute_set_intersection.cpp:193-233)
* :func:`adaptive_share_join`        — ``adaptiveShareJoin`` with the ALL_LEVEL / LOCAL_COUNT /
  COLLECT_RESULT outputs (matching/adaptive.cpp:1179-2279)

All compute runs on the GPU; there is no CPU fallback.  If the shared library
is missing, importing this package raises.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libasdm_b200.so")
BIN_DIR = os.path.join(_PKG, "bin")

OK, ERR_INVALID, ERR_IO, ERR_CUDA, ERR_OOM, ERR_OVERFLOW, ERR_TIMEOUT, ERR_CAPACITY, ERR_INTERNAL, ERR_LIMIT = range(10)
MODE_COUNT, MODE_LOCAL, MODE_EMBED = 0, 1, 2

_ERR_NAMES = {ERR_INVALID: "invalid", ERR_IO: "io", ERR_CUDA: "cuda", ERR_OOM: "oom", ERR_OVERFLOW: "overflow",
              ERR_TIMEOUT: "timeout", ERR_CAPACITY: "capacity", ERR_INTERNAL: "internal", ERR_LIMIT: "limit"}


class AsdmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("%s (%s)" % (msg, _ERR_NAMES.get(code, code)))
        self.code = code


if not os.path.exists(LIB_PATH):
    raise ImportError("libasdm_b200.so not built: run `python -m asdmatch_b200.build` (%s)" % LIB_PATH)
_lib = C.CDLL(LIB_PATH)

_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_vp = C.c_void_p


class RunOpts(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("budget_bytes", C.c_uint64), ("time_limit_s", C.c_double),
                ("local_counts", _u64p), ("embeddings", _u32p), ("emb_capacity", C.c_uint64),
                ("count_limit", C.c_uint64)]


class RunStats(C.Structure):
    _fields_ = [("count", C.c_uint64), ("emb_rows", C.c_uint64), ("intersections", C.c_uint64),
                ("list_bytes", C.c_uint64), ("tasks", C.c_uint64), ("kernel_ms", C.c_double),
                ("build_ms", C.c_double), ("build_bytes", C.c_uint64), ("tails_lane", C.c_uint64),
                ("tails_warp", C.c_uint64), ("busy_warp_ms", C.c_double), ("idle_warp_ms", C.c_double)]


def _sig(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


_last_error = _sig("asdm_last_error", C.c_char_p, [])
_version = _sig("asdm_version", C.c_char_p, [])
_hg_load = _sig("asdm_host_graph_load", C.c_int, [C.c_char_p, C.POINTER(_vp)])
_hg_from_edges = _sig("asdm_host_graph_from_edges", C.c_int, [C.c_uint32, _u32p, C.c_uint64, _u32p, C.POINTER(_vp)])
_hg_info = _sig("asdm_host_graph_info", C.c_int, [_vp, _u32p, _u64p, _u32p])
_hg_csr = _sig("asdm_host_graph_csr", C.c_int, [_vp, C.POINTER(_u32p), C.POINTER(_u32p), C.POINTER(_u32p)])
_hg_write = _sig("asdm_host_graph_write", C.c_int, [_vp, C.c_char_p])
_hg_free = _sig("asdm_host_graph_free", None, [_vp])
_hg_write_bin = _sig("asdm_host_graph_write_binary", C.c_int, [_vp, C.c_char_p])
_hg_load_bin = _sig("asdm_host_graph_load_binary", C.c_int, [C.c_char_p, C.POINTER(_vp)])
_gen_cl = _sig("asdm_gen_chung_lu", C.c_int, [C.c_uint32, C.c_uint64, C.c_double, C.c_uint32, C.c_double, C.c_uint64,
                                              C.POINTER(_vp)])
_gen_clc = _sig("asdm_gen_chung_lu_capped", C.c_int, [C.c_uint32, C.c_uint64, C.c_double, C.c_uint32, C.c_double,
                                                      C.c_double, C.c_uint64, C.POINTER(_vp)])
_gen_q = _sig("asdm_gen_query", C.c_int, [_vp, C.c_uint32, C.c_int, C.c_uint64, C.POINTER(_vp)])
_g_upload = _sig("asdm_graph_upload", C.c_int, [_u32p, _u32p, _u32p, C.c_uint32, C.c_uint64, C.c_uint32,
                                                C.POINTER(_vp)])
_g_free = _sig("asdm_graph_free", C.c_int, [_vp])
_cs_build = _sig("asdm_candidate_space", C.c_int, [_vp, _u32p, _u32p, _u32p, C.c_uint32, C.POINTER(_vp),
                                                   C.POINTER(C.c_int)])
_cs_sizes = _sig("asdm_cs_sizes", C.c_int, [_vp, _u32p])
_cs_read = _sig("asdm_cs_read", C.c_int, [_vp, C.c_uint32, _u32p, C.c_uint32])
_cs_read_edges = _sig("asdm_cs_read_edges", C.c_int, [_vp, C.c_uint32, C.c_uint32, _u32p, _u32p, C.c_uint64, _u64p])
_cs_free = _sig("asdm_cs_free", C.c_int, [_vp])
_intersect = _sig("asdm_intersect_batch", C.c_int, [_u32p, _u64p, C.c_uint64, _u32p, C.c_uint32, _u64p, _u32p, _u32p])
_plan_create = _sig("asdm_plan_create", C.c_int, [_vp, _u32p, C.POINTER(_vp)])
_plan_order = _sig("asdm_plan_order", C.c_int, [_vp, _u32p])
_plan_free = _sig("asdm_plan_free", C.c_int, [_vp])
_run_plan = _sig("asdm_run_plan", C.c_int, [_vp, _vp, C.POINTER(RunOpts), C.POINTER(RunStats)])
_count_query = _sig("asdm_count_query", C.c_int, [_vp, _u32p, _u32p, _u32p, C.c_uint32, C.POINTER(RunOpts),
                                                  C.POINTER(RunStats)])
class Tuning(C.Structure):
    _fields_ = [("enum_min_blocks", C.c_uint32), ("lane_leaf_max", C.c_uint32), ("planner", C.c_uint32),
                ("root_block_min", C.c_uint32), ("padded_cap_log2", C.c_uint32), ("merge_ratio", C.c_uint32)]


PLANNER_DP = 0
PLANNER_GREEDY = 1


_set_tuning = _sig("asdm_graph_set_tuning", C.c_int, [_vp, C.POINTER(Tuning)])
_get_tuning = _sig("asdm_graph_get_tuning", C.c_int, [_vp, C.POINTER(Tuning)])
_run_batch_local = _sig("asdm_run_batch_local", C.c_int,
                        [_vp, C.c_uint32, _u32p, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p, C.c_double, _u64p,
                         C.POINTER(C.c_int), C.POINTER(_u64p), C.POINTER(RunStats)])
_card_load = _sig("asdm_card_load", C.c_int, [C.c_char_p, C.POINTER(_vp)])
_card_create = _sig("asdm_card_create", C.c_int, [C.POINTER(_vp)])
_card_set = _sig("asdm_card_set", C.c_int, [_vp, C.c_uint64, C.c_double])
_card_lookup = _sig("asdm_card_lookup", C.c_int, [_vp, C.c_uint64, C.POINTER(C.c_double)])
_card_info = _sig("asdm_card_info", C.c_int, [_vp, _u32p, _u64p, C.POINTER(C.c_double)])
_card_write = _sig("asdm_card_write", C.c_int, [_vp, C.c_char_p, C.c_double])
_card_free = _sig("asdm_card_free", None, [_vp])
_plan_create_card = _sig("asdm_plan_create_card", C.c_int, [_vp, _vp, C.POINTER(_vp)])
_card_sample = _sig("asdm_card_sample", C.c_int, [_vp, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(_vp)])
_sample_subsets = _sig("asdm_sample_subsets", C.c_int, [_vp, C.c_uint32, _u64p, C.c_uint32, C.c_uint64,
                                                        C.POINTER(C.c_double)])
_gemm = _sig("asdm_gemm_bf16", C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16),
                                         C.POINTER(C.c_float)])
class BatchOpts(C.Structure):
    _fields_ = [("time_limit_s", C.c_double), ("count_limit", C.c_uint64), ("cards", C.POINTER(_vp)),
                ("estimator", _vp), ("learned_max_subset", C.c_uint32), ("query_time_limit_s", C.c_double)]


_run_batch_ex = _sig("asdm_run_batch_ex", C.c_int,
                     [_vp, C.c_uint32, _u32p, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p, C.POINTER(BatchOpts), _u64p,
                      C.POINTER(C.c_int), C.POINTER(_u64p), C.POINTER(RunStats)])
_cs_edge_totals = _sig("asdm_cs_edge_totals", C.c_int, [_vp, _u64p])
_cs_lower_bound = _sig("asdm_cs_count_lower_bound", C.c_int, [_vp, _u64p, C.POINTER(C.c_int)])
_cs_digest = _sig("asdm_cs_digest", C.c_int, [_vp, _u64p, _u32p])
CS_TWO_SCAN, CS_LABEL_RUNS = 1, 2
_est_create = _sig("asdm_est_create", C.c_int, [C.c_uint32, C.c_uint64, C.POINTER(_vp)])
_est_train = _sig("asdm_est_train_step", C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_float), _u32p, _u32p, _u32p,
                                                   C.POINTER(C.c_float), C.c_float, C.POINTER(C.c_float)])
_est_predict = _sig("asdm_est_predict", C.c_int, [_vp, C.c_int, C.c_int, C.POINTER(C.c_float), _u32p, _u32p, _u32p,
                                                  C.POINTER(C.c_float)])
_est_params = _sig("asdm_est_params", C.c_int, [_vp, C.POINTER(C.c_float), C.c_uint64, _u64p])
_est_set_params = _sig("asdm_est_set_params", C.c_int, [_vp, C.POINTER(C.c_float), C.c_uint64])
_est_free = _sig("asdm_est_free", None, [_vp])
_prefix_counts = _sig("asdm_prefix_counts", C.c_int, [_vp, C.c_uint32, _u32p, _u32p, C.c_double, C.c_uint64, _u64p,
                                                      C.POINTER(C.c_int)])
_cs_batch = _sig("asdm_candidate_space_batch", C.c_int, [_vp, C.c_uint32, _u32p, _u64p, _u32p, _u64p, _u32p, _u64p,
                                                         _u32p, C.POINTER(_vp), C.POINTER(C.c_int), C.POINTER(C.c_int)])
_run_planned = _sig("asdm_run_planned", C.c_int, [C.c_uint32, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(BatchOpts),
                                                  _u64p, C.POINTER(C.c_int), C.POINTER(RunStats)])
EST_FEATURES = 44
_est_features = _sig("asdm_est_features", C.c_int, [_vp, C.c_uint32, _u64p, C.POINTER(C.c_float), _u32p, _u32p,
                                                    C.c_uint64, _u32p, _u64p, _u64p])
_plan_learned = _sig("asdm_plan_create_learned", C.c_int, [C.c_uint32, C.POINTER(_vp), _vp, C.c_uint32,
                                                           C.POINTER(_vp)])
_run_planned_profile = _sig("asdm_run_planned_profile", C.c_int,
                            [C.c_uint32, C.POINTER(_vp), C.POINTER(_vp), C.POINTER(BatchOpts), _u64p,
                             C.POINTER(C.c_int), C.POINTER(RunStats), _u64p])
_launches = _sig("asdm_kernel_launches", C.c_uint64, [])
_g_stream = _sig("asdm_graph_stream", C.c_int, [_vp, C.POINTER(_vp)])
_cs_stats = _sig("asdm_cs_stats", C.c_int, [_vp, _u64p, C.POINTER(C.c_double)])
_run_batch = _sig("asdm_run_batch", C.c_int, [_vp, C.c_uint32, _u32p, _u64p, _u32p, _u64p, _u32p, _u64p, _u32p,
                                              C.c_double, _u64p, C.POINTER(C.c_int), C.POINTER(RunStats)])


def _check(rc: int, what: str = ""):
    if rc != OK:
        msg = (_last_error() or b"").decode(errors="replace")
        raise AsdmError(rc, ("%s: %s" % (what, msg)) if what else msg)


def _ptr(a: np.ndarray, ty=_u32p):
    return a.ctypes.data_as(ty)


def version() -> str:
    return _version().decode()


def to_bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 bit patterns (uint16)."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def from_bf16_bits(b: np.ndarray) -> np.ndarray:
    return (np.asarray(b, np.uint32) << 16).view(np.float32)


def gemm_bf16(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """C = A @ B^T on the tcgen05 tensor cores (A: M x K, B: N x K, bf16 inputs, fp32 out)."""
    M, K = a.shape
    N = b.shape[0]
    ab, bb = to_bf16_bits(a), to_bf16_bits(b)
    c = np.zeros((M, N), np.float32)
    _check(_gemm(M, N, K, ab.ctypes.data_as(C.POINTER(C.c_uint16)), bb.ctypes.data_as(C.POINTER(C.c_uint16)),
                 c.ctypes.data_as(C.POINTER(C.c_float))), "gemm")
    return c


def kernel_launches() -> int:
    """Kernels the library has launched so far in this process."""
    return int(_launches())


class HostGraph:
    """Host CSR in the reference's layout: neighbours sorted by (label, id)."""

    def __init__(self, handle):
        self._h = _vp(handle)
        n, m2, nl = C.c_uint32(), C.c_uint64(), C.c_uint32()
        _check(_hg_info(self._h, C.byref(n), C.byref(m2), C.byref(nl)))
        self.n, self.m2, self.nlabels = n.value, m2.value, nl.value
        o, b, l = _u32p(), _u32p(), _u32p()
        _check(_hg_csr(self._h, C.byref(o), C.byref(b), C.byref(l)))
        # zero-copy views, valid while this object lives
        self.offsets = np.ctypeslib.as_array(o, shape=(self.n + 1,)) if self.n + 1 else np.zeros(1, np.uint32)
        self.nbrs = np.ctypeslib.as_array(b, shape=(self.m2,)) if self.m2 else np.zeros(0, np.uint32)
        self.labels = np.ctypeslib.as_array(l, shape=(self.n,)) if self.n else np.zeros(0, np.uint32)

    @classmethod
    def load(cls, path: str) -> "HostGraph":
        h = _vp()
        _check(_hg_load(path.encode(), C.byref(h)), path)
        return cls(h.value)

    @classmethod
    def from_edges(cls, n: int, labels: Sequence[int], edges) -> "HostGraph":
        lab = np.ascontiguousarray(labels, dtype=np.uint32)
        e = np.ascontiguousarray(np.asarray(edges, dtype=np.uint32).reshape(-1))
        h = _vp()
        _check(_hg_from_edges(n, _ptr(lab), len(e) // 2, _ptr(e), C.byref(h)), "from_edges")
        return cls(h.value)

    @classmethod
    def chung_lu(cls, n: int, m: int, gamma: float, nlabels: int, zipf_s: float, seed: int,
                 wmax: float = 0.0) -> "HostGraph":
        """Seeded Chung-Lu graph; wmax is the largest expected degree (0: sqrt(2m))."""
        h = _vp()
        if wmax > 0:
            _check(_gen_clc(n, m, gamma, nlabels, zipf_s, wmax, seed, C.byref(h)), "chung_lu")
        else:
            _check(_gen_cl(n, m, gamma, nlabels, zipf_s, seed, C.byref(h)), "chung_lu")
        return cls(h.value)

    def random_walk_query(self, size: int, seed: int, density: int = 0) -> "HostGraph":
        """density: 0 any, 1 dense (avg degree >= 3), 2 sparse (< 3)."""
        h = _vp()
        _check(_gen_q(self._h, size, density, seed, C.byref(h)), "query")
        return HostGraph(h.value)

    def write(self, path: str):
        _check(_hg_write(self._h, path.encode()), path)

    def write_binary(self, path: str):
        """The reference's binary graph cache (Graph::writeToStream)."""
        _check(_hg_write_bin(self._h, path.encode()), path)

    @classmethod
    def load_binary(cls, path: str) -> "HostGraph":
        """Graph::readFromStream (relation/graph.cpp:293-314)."""
        h = _vp()
        _check(_hg_load_bin(path.encode(), C.byref(h)), path)
        return cls(h.value)

    def degree(self, v: int) -> int:
        return int(self.offsets[v + 1] - self.offsets[v])

    def edges(self) -> np.ndarray:
        src = np.repeat(np.arange(self.n, dtype=np.uint32), np.diff(self.offsets.astype(np.int64)))
        keep = src < self.nbrs
        return np.stack([src[keep], self.nbrs[keep]], axis=1)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _hg_free is not None:  # module globals are gone at interpreter exit
            _hg_free(h)
            self._h = _vp()


def load_graph_from_text_file(path: str) -> HostGraph:
    """Graph::loadGraphFromTextFile (relation/graph.cpp:68-148)."""
    return HostGraph.load(path)


class DeviceGraph:
    """Data graph resident in HBM (CSR + label-run index)."""

    def __init__(self, g: HostGraph):
        h = _vp()
        _check(_g_upload(_ptr(g.offsets), _ptr(g.nbrs), _ptr(g.labels), g.n, g.m2, max(g.nlabels, 1), C.byref(h)),
               "upload")
        self._h = h
        self.n = g.n
        self.host = g
        # candidate spaces built on this graph: they free their device memory
        # on the graph's stream, so they are closed before the graph is
        self._spaces = weakref.WeakSet()

    def set_tuning(self, enum_min_blocks: int, lane_leaf_max: int, planner: Optional[int] = None,
                   root_block_min: Optional[int] = None, padded_cap_log2: Optional[int] = None,
                   merge_ratio: Optional[int] = None):
        cur = self.tuning()
        planner = cur["planner"] if planner is None else planner
        root_block_min = cur["root_block_min"] if root_block_min is None else root_block_min
        padded_cap_log2 = cur["padded_cap_log2"] if padded_cap_log2 is None else padded_cap_log2
        merge_ratio = cur["merge_ratio"] if merge_ratio is None else merge_ratio
        _check(_set_tuning(self._h, C.byref(Tuning(enum_min_blocks, lane_leaf_max, planner, root_block_min,
                                                   padded_cap_log2, merge_ratio))), "tuning")

    def tuning(self):
        t = Tuning()
        _check(_get_tuning(self._h, C.byref(t)))
        return {"enum_min_blocks": t.enum_min_blocks, "lane_leaf_max": t.lane_leaf_max, "planner": t.planner,
                "root_block_min": t.root_block_min, "padded_cap_log2": t.padded_cap_log2,
                "merge_ratio": t.merge_ratio}

    def stream(self) -> int:
        """cudaStream_t (as an int) the library uses for this graph."""
        s = _vp()
        _check(_g_stream(self._h, C.byref(s)))
        return s.value or 0

    def close(self):
        for cs in list(getattr(self, "_spaces", ())):
            try:
                cs.close()
            except Exception:
                pass
        if self._h is not None and self._h.value:
            _g_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class CandidateSpace:
    """CFL candidate space on the device (CandidateSpace::buildCandCFL)."""

    def __init__(self, dg: DeviceGraph, q: HostGraph):
        h = _vp()
        ne = C.c_int()
        _check(_cs_build(dg._h, _ptr(q.offsets), _ptr(q.nbrs), _ptr(q.labels), q.n, C.byref(h), C.byref(ne)),
               "candidate space")
        self._h = h
        self.q = q
        self.dg = dg
        self.nonempty = bool(ne.value)
        dg._spaces.add(self)

    def build_cand_cfl(self) -> bool:
        """The reference's return value: False when some candidate set is empty."""
        return self.nonempty

    def edge_totals(self) -> np.ndarray:
        """Candidate-edge entries per directed query edge, query-CSR order."""
        out = np.zeros(max(int(self.q.offsets[-1]), 1), np.uint64)
        _check(_cs_edge_totals(self._h, _ptr(out, _u64p)))
        return out[:int(self.q.offsets[-1])]

    def digest(self):
        """(digest, flags): a device-computed 64-bit digest of C(u) and the
        candidate-edge lists, and the CS_* bits of how they were built."""
        d = C.c_uint64()
        f = C.c_uint32()
        _check(_cs_digest(self._h, C.byref(d), C.byref(f)), "digest")
        return int(d.value), int(f.value)

    def sample_cardinalities(self, masks: Sequence[int], walks: int = 0, seed: int = 0) -> np.ndarray:
        """Sampling estimates of the partial-match counts of connected vertex
        subsets (asdm_sample_subsets)."""
        m = np.ascontiguousarray(masks, dtype=np.uint64)
        out = np.zeros(max(len(m), 1), np.float64)
        _check(_sample_subsets(self._h, len(m), _ptr(m, _u64p), walks, seed,
                               out.ctypes.data_as(C.POINTER(C.c_double))), "sample")
        return out[:len(m)]

    def count_lower_bound(self):
        """(bound, exceeds): a lower bound of the embedding count (capped at
        2^64 - 1) and whether it shows the count is at least 2^64."""
        lb = C.c_uint64()
        ex = C.c_int()
        _check(_cs_lower_bound(self._h, C.byref(lb), C.byref(ex)), "lower bound")
        return int(lb.value), bool(ex.value)

    def prefix_counts(self, orders: Sequence[Sequence[int]], time_limit_s: float = 0.0, count_limit: int = 0):
        """Partial-match counts of each prefix (a connected sequence of query
        vertices) inside this candidate space, in one batched launch.
        Returns (counts uint64, status int32)."""
        n = self.q.n
        k = len(orders)
        mat = np.zeros((max(k, 1), n), np.uint32)
        depths = np.zeros(max(k, 1), np.uint32)
        for i, o in enumerate(orders):
            mat[i, :len(o)] = o
            depths[i] = len(o)
        counts = np.zeros(max(k, 1), np.uint64)
        status = np.zeros(max(k, 1), np.int32)
        rc = _prefix_counts(self._h, k, _ptr(mat), _ptr(depths), time_limit_s, count_limit, _ptr(counts, _u64p),
                            status.ctypes.data_as(C.POINTER(C.c_int)))
        if rc == ERR_CUDA:
            _check(rc, "prefix counts")
        return counts[:k], status[:k]

    @classmethod
    def _wrap(cls, h: int, q: HostGraph, dg: DeviceGraph, nonempty: bool) -> "CandidateSpace":
        obj = cls.__new__(cls)
        obj._h = _vp(h)
        obj.q = q
        obj.dg = dg
        obj.nonempty = nonempty
        dg._spaces.add(obj)
        return obj

    def build_stats(self):
        """(algorithmic bytes, device ms) of the candidate-space build."""
        b, ms = C.c_uint64(), C.c_double()
        _check(_cs_stats(self._h, C.byref(b), C.byref(ms)))
        return b.value, ms.value

    def sizes(self) -> np.ndarray:
        out = np.zeros(self.q.n, np.uint32)
        _check(_cs_sizes(self._h, _ptr(out)))
        return out

    def candidate_set(self, u: int) -> np.ndarray:
        n = int(self.sizes()[u])
        out = np.zeros(max(n, 1), np.uint32)
        _check(_cs_read(self._h, u, _ptr(out), n))
        return out[:n]

    def candidate_edge(self, u: int, u2: int):
        """(offsets, neighbour ids) of candidateEdge[u][v][u2] for v in C(u)."""
        n = int(self.sizes()[u])
        off = np.zeros(n + 1, np.uint32)
        total = C.c_uint64()
        # first call with capacity 0 only learns the size
        rc = _cs_read_edges(self._h, u, u2, _ptr(off), None, 0, C.byref(total))
        if rc not in (OK, ERR_CAPACITY):
            _check(rc)
        vals = np.zeros(max(total.value, 1), np.uint32)
        _check(_cs_read_edges(self._h, u, u2, _ptr(off), _ptr(vals), total.value, C.byref(total)))
        return off, vals[:total.value]

    def write_to_stream(self) -> str:
        """Text dump: 'C u n v...' lines, then CandidateSpace::writeToStream (candidate_space.cpp:489-505)."""
        q = self.q
        lines = []
        for u in range(q.n):
            c = self.candidate_set(u)
            lines.append("C %d %d%s" % (u, len(c), "".join(" %d" % v for v in c)))
        for u in range(q.n):
            c = self.candidate_set(u)
            for e in range(int(q.offsets[u]), int(q.offsets[u + 1])):
                u2 = int(q.nbrs[e])
                lines.append("# %d %d" % (u, u2))
                off, vals = self.candidate_edge(u, u2)
                for i, v in enumerate(c):
                    for w in vals[off[i]:off[i + 1]]:
                        lines.append("%d %d" % (v, w))
        return "\n".join(lines) + "\n"

    def close(self):
        if self._h is not None and self._h.value:
            _cs_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Card:
    """The .card plan cache: subset bitmask (bit u = query vertex u) -> cardinality."""

    def __init__(self, path: Optional[str] = None):
        h = _vp()
        if path is None:
            _check(_card_create(C.byref(h)))
        else:
            _check(_card_load(path.encode(), C.byref(h)), path)
        self._h = h

    def info(self):
        b, e, t = C.c_uint32(), C.c_uint64(), C.c_double()
        _check(_card_info(self._h, C.byref(b), C.byref(e), C.byref(t)))
        return {"bags": b.value, "entries": e.value, "plan_seconds": t.value}

    def __setitem__(self, subset: int, card: float):
        _check(_card_set(self._h, subset, card))

    def __getitem__(self, subset: int) -> float:
        v = C.c_double()
        _check(_card_lookup(self._h, subset, C.byref(v)))
        return v.value

    def write(self, path: str, plan_seconds: float = 0.0):
        _check(_card_write(self._h, path.encode(), plan_seconds), path)

    @classmethod
    def sample(cls, cs: "CandidateSpace", max_subset: int = 0, walks: int = 0, seed: int = 0) -> "Card":
        """Sampling estimates of the query's connected sub-queries of 3..max_subset
        vertices, made on the device (asdm_card_sample)."""
        h = _vp()
        _check(_card_sample(cs._h, max_subset, walks, seed, C.byref(h)), "sample")
        c = cls.__new__(cls)
        c._h = h
        return c

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _card_free is not None:  # module globals are gone at interpreter exit
            _card_free(h)
            self._h = None


class Plan:
    def __init__(self, cs: CandidateSpace, order: Optional[Sequence[int]] = None, card: Optional[Card] = None):
        h = _vp()
        o = None
        if order is not None:
            arr = np.ascontiguousarray(order, dtype=np.uint32)
            o = _ptr(arr)
        if card is not None:
            _check(_plan_create_card(cs._h, card._h, C.byref(h)), "plan")
            self._h = h
            self.n = cs.q.n
            return
        _check(_plan_create(cs._h, o, C.byref(h)), "plan")
        self._h = h
        self.n = cs.q.n

    def order(self) -> List[int]:
        out = np.zeros(self.n, np.uint32)
        _check(_plan_order(self._h, _ptr(out)))
        return out.tolist()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _plan_free is not None:  # module globals are gone at interpreter exit
            _plan_free(h)
            self._h = None


@dataclass
class MatchResult:
    count: int
    local_counts: Optional[np.ndarray] = None   # |Vg| x |Vq| uint64
    embeddings: Optional[np.ndarray] = None     # rows x |Vq| uint32, lexicographically sorted
    intersections: int = 0
    list_bytes: int = 0
    tasks: int = 0
    kernel_ms: float = 0.0
    nonempty: bool = True


def adaptive_share_join(cs: CandidateSpace, plan: Optional[Plan] = None, mode: int = MODE_COUNT,
                        emb_capacity: int = 0, budget_bytes: int = 0, time_limit_s: float = 0.0,
                        count_limit: int = 0) -> MatchResult:
    """Exact enumeration of one query: count, local counts (MODE_LOCAL), embeddings (MODE_EMBED)."""
    n = cs.q.n
    opts = RunOpts()
    opts.mode = mode
    opts.budget_bytes = budget_bytes
    opts.time_limit_s = time_limit_s
    opts.count_limit = count_limit
    local = emb = None
    if mode & MODE_LOCAL:
        local = np.zeros((cs.dg.n, n), np.uint64)
        opts.local_counts = _ptr(local, _u64p)
    if mode & MODE_EMBED:
        emb = np.zeros((max(emb_capacity, 1), n), np.uint32)
        opts.embeddings = _ptr(emb)
        opts.emb_capacity = emb_capacity
    st = RunStats()
    if cs.nonempty and plan is None:
        plan = Plan(cs)
    _check(_run_plan(cs._h, plan._h if plan is not None else None, C.byref(opts), C.byref(st)), "run")
    if emb is not None:
        emb = emb[:st.emb_rows]
    return MatchResult(st.count, local, emb, st.intersections, st.list_bytes, st.tasks, st.kernel_ms, cs.nonempty)


def match(dg: DeviceGraph, q: HostGraph, mode: int = MODE_COUNT, order: Optional[Sequence[int]] = None,
          time_limit_s: float = 0.0) -> MatchResult:
    """Candidate space + plan + enumeration for one query; embeddings sized by a counting pass."""
    cs = CandidateSpace(dg, q)
    try:
        if not cs.nonempty:
            local = np.zeros((dg.n, q.n), np.uint64) if mode & MODE_LOCAL else None
            emb = np.zeros((0, q.n), np.uint32) if mode & MODE_EMBED else None
            return MatchResult(0, local, emb, nonempty=False)
        plan = Plan(cs, order)
        cap = 0
        if mode & MODE_EMBED:
            cap = adaptive_share_join(cs, plan, MODE_COUNT, time_limit_s=time_limit_s).count
        return adaptive_share_join(cs, plan, mode, emb_capacity=cap, time_limit_s=time_limit_s)
    finally:
        cs.close()


def count_query(dg: DeviceGraph, q: HostGraph, time_limit_s: float = 0.0, count_limit: int = 0) -> MatchResult:
    """One-call count (asdm_count_query)."""
    opts = RunOpts()
    opts.mode = MODE_COUNT
    opts.time_limit_s = time_limit_s
    opts.count_limit = count_limit
    st = RunStats()
    _check(_count_query(dg._h, _ptr(q.offsets), _ptr(q.nbrs), _ptr(q.labels), q.n, C.byref(opts), C.byref(st)),
           "count")
    return MatchResult(st.count, intersections=st.intersections, list_bytes=st.list_bytes, tasks=st.tasks,
                       kernel_ms=st.kernel_ms)


def leapfrog_join(lists_per_set: Sequence[Sequence[np.ndarray]]) -> List[np.ndarray]:
    """Batched k-way sorted intersection on the device (LeapfrogJoin)."""
    vals, loff, first, ooff = [], [0], [0], [0]
    for lists in lists_per_set:
        mn = 0
        for l in lists:
            a = np.ascontiguousarray(l, dtype=np.uint32)
            vals.append(a)
            loff.append(loff[-1] + len(a))
        if lists:
            mn = min(len(l) for l in lists)
        first.append(first[-1] + len(lists))
        ooff.append(ooff[-1] + mn)
    values = np.concatenate(vals) if vals else np.zeros(1, np.uint32)
    if len(values) == 0:
        values = np.zeros(1, np.uint32)
    loff_a = np.asarray(loff, np.uint64)
    first_a = np.asarray(first, np.uint32)
    ooff_a = np.asarray(ooff, np.uint64)
    out = np.zeros(max(int(ooff_a[-1]), 1), np.uint32)
    cnt = np.zeros(max(len(lists_per_set), 1), np.uint32)
    _check(_intersect(_ptr(values), _ptr(loff_a, _u64p), len(loff) - 1, _ptr(first_a), len(lists_per_set),
                      _ptr(ooff_a, _u64p), _ptr(out), _ptr(cnt)), "intersect")
    return [out[ooff[i]:ooff[i] + cnt[i]].copy() for i in range(len(lists_per_set))]


class BatchInput:
    """Queries packed once into the host arrays asdm_run_batch takes."""

    def __init__(self, queries: Sequence[HostGraph]):
        self.nq = len(queries)
        self.sizes = np.asarray([q.n for q in queries], np.uint32)
        self.offs = np.concatenate([q.offsets for q in queries]).astype(np.uint32)
        self.nbrs = np.concatenate([q.nbrs for q in queries] + [np.zeros(1, np.uint32)]).astype(np.uint32)
        self.labs = np.concatenate([q.labels for q in queries]).astype(np.uint32)
        self.ob = np.cumsum([0] + [q.n + 1 for q in queries[:-1]]).astype(np.uint64)
        self.nb = np.cumsum([0] + [q.m2 for q in queries[:-1]]).astype(np.uint64)
        self.lb = np.cumsum([0] + [q.n for q in queries[:-1]]).astype(np.uint64)
        self.counts = np.zeros(self.nq, np.uint64)
        self.status = np.zeros(self.nq, np.int32)

    def nbytes(self):
        return int(self.sizes.nbytes + self.offs.nbytes + self.nbrs.nbytes + self.labs.nbytes + self.ob.nbytes +
                   self.nb.nbytes + self.lb.nbytes)


def run_batch_packed(dg: DeviceGraph, b: BatchInput, time_limit_s: float = 0.0) -> RunStats:
    """Batched counting of pre-packed queries; results land in b.counts / b.status."""
    st = RunStats()
    rc = _run_batch(dg._h, b.nq, _ptr(b.sizes), _ptr(b.ob, _u64p), _ptr(b.offs), _ptr(b.nb, _u64p), _ptr(b.nbrs),
                    _ptr(b.lb, _u64p), _ptr(b.labs), time_limit_s, _ptr(b.counts, _u64p),
                    b.status.ctypes.data_as(C.POINTER(C.c_int)), C.byref(st))
    if rc == ERR_CUDA:
        _check(rc, "batch")
    return st


def run_batch_local(dg: DeviceGraph, queries: Sequence[HostGraph], time_limit_s: float = 0.0):
    """Batched LOCAL_COUNT: returns (counts, status, [|Vg| x |Vq_i| uint64 matrices])."""
    b = BatchInput(queries)
    mats = [np.zeros((dg.n, q.n), np.uint64) for q in queries]
    ptrs = (_u64p * max(1, len(mats)))(*[_ptr(m, _u64p) for m in mats])
    st = RunStats()
    rc = _run_batch_local(dg._h, b.nq, _ptr(b.sizes), _ptr(b.ob, _u64p), _ptr(b.offs), _ptr(b.nb, _u64p), _ptr(b.nbrs),
                          _ptr(b.lb, _u64p), _ptr(b.labs), time_limit_s, _ptr(b.counts, _u64p),
                          b.status.ctypes.data_as(C.POINTER(C.c_int)), ptrs, C.byref(st))
    if rc == ERR_CUDA:
        _check(rc, "batch")
    return b.counts.copy(), b.status.copy(), mats


def run_batch_ex(dg: DeviceGraph, b: BatchInput, time_limit_s: float = 0.0, count_limit: int = 0,
                 cards: Optional[Sequence[Optional["Card"]]] = None, estimator: Optional["Estimator"] = None,
                 learned_max_subset: int = 0, query_time_limit_s: float = 0.0) -> RunStats:
    """Batched counting with per-query count limits, per-query GPU-time
    budgets (query_time_limit_s: the time a query may take as if it ran alone
    on the GPU; past it that query alone reports ERR_TIMEOUT), plan caches or
    learned plans; results in b.counts / b.status."""
    opts = BatchOpts()
    opts.time_limit_s = time_limit_s
    opts.count_limit = count_limit
    opts.query_time_limit_s = query_time_limit_s
    if estimator is not None:
        opts.estimator = estimator._h
        opts.learned_max_subset = learned_max_subset
    keep = None
    if cards is not None:
        keep = (_vp * max(1, b.nq))(*[(c._h if c is not None else _vp()) for c in cards])
        opts.cards = C.cast(keep, C.POINTER(_vp))
    st = RunStats()
    rc = _run_batch_ex(dg._h, b.nq, _ptr(b.sizes), _ptr(b.ob, _u64p), _ptr(b.offs), _ptr(b.nb, _u64p), _ptr(b.nbrs),
                       _ptr(b.lb, _u64p), _ptr(b.labs), C.byref(opts), _ptr(b.counts, _u64p),
                       b.status.ctypes.data_as(C.POINTER(C.c_int)), None, C.byref(st))
    if rc == ERR_CUDA:
        _check(rc, "batch")
    return st


def run_batch_local_ex(dg: DeviceGraph, queries: Sequence[HostGraph], time_limit_s: float = 0.0,
                       query_time_limit_s: float = 0.0):
    """Batched LOCAL_COUNT with per-query GPU-time budgets: (counts, status,
    [|Vg| x |Vq_i| uint64 matrices], RunStats); a query's matrix is valid when
    its status is OK."""
    b = BatchInput(queries)
    mats = [np.zeros((dg.n, q.n), np.uint64) for q in queries]
    ptrs = (_u64p * max(1, len(mats)))(*[_ptr(m, _u64p) for m in mats])
    opts = BatchOpts()
    opts.time_limit_s = time_limit_s
    opts.query_time_limit_s = query_time_limit_s
    st = RunStats()
    rc = _run_batch_ex(dg._h, b.nq, _ptr(b.sizes), _ptr(b.ob, _u64p), _ptr(b.offs), _ptr(b.nb, _u64p), _ptr(b.nbrs),
                       _ptr(b.lb, _u64p), _ptr(b.labs), C.byref(opts), _ptr(b.counts, _u64p),
                       b.status.ctypes.data_as(C.POINTER(C.c_int)), ptrs, C.byref(st))
    if rc == ERR_CUDA:
        _check(rc, "batch")
    return b.counts.copy(), b.status.copy(), mats, st


def candidate_spaces(dg: DeviceGraph, queries: Sequence[HostGraph], b: Optional[BatchInput] = None):
    """Candidate spaces of many queries built in groups; None where a build failed."""
    b = b or BatchInput(queries)
    nq = b.nq
    hs = (_vp * max(1, nq))()
    ne = np.zeros(max(1, nq), np.int32)
    st = np.zeros(max(1, nq), np.int32)
    rc = _cs_batch(dg._h, nq, _ptr(b.sizes), _ptr(b.ob, _u64p), _ptr(b.offs), _ptr(b.nb, _u64p), _ptr(b.nbrs),
                   _ptr(b.lb, _u64p), _ptr(b.labs), hs, ne.ctypes.data_as(C.POINTER(C.c_int)),
                   st.ctypes.data_as(C.POINTER(C.c_int)))
    if rc == ERR_CUDA:
        _check(rc, "candidate spaces")
    return [CandidateSpace._wrap(hs[i], queries[i], dg, bool(ne[i])) if st[i] == OK and hs[i] else None
            for i in range(nq)]


def run_planned(css: Sequence[CandidateSpace], plans: Sequence[Optional["Plan"]], time_limit_s: float = 0.0,
                count_limit: int = 0, query_time_limit_s: float = 0.0):
    """One persistent launch over given candidate spaces and plans: (counts, status, RunStats)."""
    nq = len(css)
    ch = (_vp * max(1, nq))(*[c._h for c in css])
    ph = (_vp * max(1, nq))(*[(p._h if p is not None else _vp()) for p in plans])
    opts = BatchOpts()
    opts.time_limit_s = time_limit_s
    opts.count_limit = count_limit
    opts.query_time_limit_s = query_time_limit_s
    counts = np.zeros(max(1, nq), np.uint64)
    status = np.zeros(max(1, nq), np.int32)
    st = RunStats()
    rc = _run_planned(nq, ch, ph, C.byref(opts), _ptr(counts, _u64p), status.ctypes.data_as(C.POINTER(C.c_int)),
                      C.byref(st))
    if rc == ERR_CUDA:
        _check(rc, "planned batch")
    return counts[:nq], status[:nq], st


def subset_features(cs: CandidateSpace, masks: Sequence[int]):
    """The estimator's input for sub-queries (vertex bitmasks) of cs's query:
    (x [nodes, EST_FEATURES] float32, adj_off, adj, node_graph)."""
    m = np.ascontiguousarray(masks, np.uint64)
    nn, na = C.c_uint64(), C.c_uint64()
    _check(_est_features(cs._h, len(m), _ptr(m, _u64p), None, None, None, 0, None, C.byref(nn), C.byref(na)),
           "features")
    x = np.zeros((max(nn.value, 1), EST_FEATURES), np.float32)
    off = np.zeros(nn.value + 1, np.uint32)
    adj = np.zeros(max(na.value, 1), np.uint32)
    gid = np.zeros(max(nn.value, 1), np.uint32)
    _check(_est_features(cs._h, len(m), _ptr(m, _u64p), x.ctypes.data_as(C.POINTER(C.c_float)), _ptr(off), _ptr(adj),
                         adj.size, _ptr(gid), C.byref(nn), C.byref(na)), "features")
    return x[:nn.value], off, adj[:na.value], gid[:nn.value]


def plans_learned(css: Sequence[CandidateSpace], est: "Estimator", max_subset: int = 0) -> List["Plan"]:
    """Plans from learned cardinalities, all queries planned in lockstep."""
    nq = len(css)
    ch = (_vp * max(1, nq))(*[c._h for c in css])
    out = (_vp * max(1, nq))()
    _check(_plan_learned(nq, ch, est._h, max_subset, out), "learned plans")
    plans = []
    for i in range(nq):
        p = Plan.__new__(Plan)
        p._h = _vp(out[i])
        p.n = css[i].q.n
        plans.append(p)
    return plans


def run_planned_profile(css: Sequence[CandidateSpace], plans: Sequence[Optional["Plan"]], time_limit_s: float = 0.0):
    """run_planned, also returning per query the SM cycles warps spent on it: (counts, status, stats, cycles)."""
    nq = len(css)
    ch = (_vp * max(1, nq))(*[c._h for c in css])
    ph = (_vp * max(1, nq))(*[(p._h if p is not None else _vp()) for p in plans])
    opts = BatchOpts()
    opts.time_limit_s = time_limit_s
    counts = np.zeros(max(1, nq), np.uint64)
    status = np.zeros(max(1, nq), np.int32)
    cycles = np.zeros(max(1, nq), np.uint64)
    st = RunStats()
    rc = _run_planned_profile(nq, ch, ph, C.byref(opts), _ptr(counts, _u64p), status.ctypes.data_as(C.POINTER(C.c_int)),
                              C.byref(st), _ptr(cycles, _u64p))
    if rc == ERR_CUDA:
        _check(rc, "planned batch")
    return counts[:nq], status[:nq], st, cycles[:nq]


class Estimator:
    """The learned cardinality estimator: a 3-layer message-passing network on
    the device (BF16 tcgen05 GEMMs, FP32 accumulation), predicting
    log(1 + cardinality) of a (sub-)query graph from per-node features."""

    def __init__(self, in_features: int, seed: int = 0):
        h = _vp()
        _check(_est_create(in_features, seed, C.byref(h)), "estimator")
        self._h = h
        self.in_features = in_features

    @staticmethod
    def _batch(x, adj_off, adj, node_graph):
        x = np.ascontiguousarray(x, np.float32)
        adj_off = np.ascontiguousarray(adj_off, np.uint32)
        adj = np.ascontiguousarray(adj if len(adj) else np.zeros(1), np.uint32)
        node_graph = np.ascontiguousarray(node_graph, np.uint32)
        return x, adj_off, adj, node_graph

    def train_step(self, x, adj_off, adj, node_graph, target, lr: float = 1e-3) -> float:
        x, adj_off, adj, node_graph = self._batch(x, adj_off, adj, node_graph)
        t = np.ascontiguousarray(target, np.float32)
        loss = C.c_float()
        _check(_est_train(self._h, x.shape[0], len(t), x.ctypes.data_as(C.POINTER(C.c_float)), _ptr(adj_off),
                          _ptr(adj), _ptr(node_graph), t.ctypes.data_as(C.POINTER(C.c_float)), lr, C.byref(loss)),
               "estimator step")
        return loss.value

    def predict(self, x, adj_off, adj, node_graph, n_graphs: int) -> np.ndarray:
        x, adj_off, adj, node_graph = self._batch(x, adj_off, adj, node_graph)
        out = np.zeros(n_graphs, np.float32)
        _check(_est_predict(self._h, x.shape[0], n_graphs, x.ctypes.data_as(C.POINTER(C.c_float)), _ptr(adj_off),
                            _ptr(adj), _ptr(node_graph), out.ctypes.data_as(C.POINTER(C.c_float))), "estimator")
        return out

    def params(self) -> np.ndarray:
        cnt = C.c_uint64()
        _check(_est_params(self._h, None, 0, C.byref(cnt)))
        out = np.zeros(cnt.value, np.float32)
        _check(_est_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float)), cnt.value, C.byref(cnt)))
        return out

    def set_params(self, p: np.ndarray):
        p = np.ascontiguousarray(p, np.float32)
        _check(_est_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float)), p.size), "estimator params")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value and _est_free is not None:  # module globals are gone at interpreter exit
            _est_free(h)
            self._h = None


def run_batch(dg: DeviceGraph, queries: Sequence[HostGraph], time_limit_s: float = 0.0):
    """Counts for many queries against one resident graph; returns (counts, status)."""
    b = BatchInput(queries)
    run_batch_packed(dg, b, time_limit_s)
    return b.counts.copy(), b.status.copy()


def autotune(dg: DeviceGraph, batch: BatchInput, reps: int = 2,
             min_blocks=(1, 3, 4, 5), lane_leaf=(32, 96, 256), planners=(PLANNER_DP, PLANNER_GREEDY),
             root_blocks=(16, 64, 256), merge_ratios=(0, 2, 8, 32), run=None):
    """Times the caller's batch under every kernel configuration (with the
    graph's current planner, root-block size and merge ratio), then every
    planner, then every smallest root-block size, then every merge/gallop
    ratio with the fastest settings so far, and keeps the fastest on `dg`
    (device time between CUDA events on the library's stream).
    `run(dg, batch)` is the timed call (default: run_batch_packed).  Returns
    (best, table)."""
    import torch
    run = run or run_batch_packed
    stream = torch.cuda.ExternalStream(dg.stream())
    want = None
    table = []

    def measure(mb, ll, pl, rb, mr):
        nonlocal want
        dg.set_tuning(mb, ll, pl, rb, merge_ratio=mr)
        run(dg, batch)  # warm
        ok = batch.status == OK
        if want is None:
            want = (batch.counts.copy(), ok.copy())
        elif not np.array_equal(batch.counts[ok & want[1]], want[0][ok & want[1]]):
            raise AsdmError(ERR_INTERNAL, "tuning changed a count")
        times = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            run(dg, batch)
            e1.record(stream)
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
        table.append({"enum_min_blocks": mb, "lane_leaf_max": ll, "planner": pl, "root_block_min": rb,
                      "merge_ratio": mr, "ms": min(times)})

    t0 = dg.tuning()
    pl0, rb0, mr0 = t0["planner"], t0["root_block_min"], t0["merge_ratio"]
    for mb in min_blocks:
        for ll in lane_leaf:
            measure(mb, ll, pl0, rb0, mr0)
    best = min(table, key=lambda r: r["ms"])
    for pl in planners:
        if pl != pl0:
            measure(best["enum_min_blocks"], best["lane_leaf_max"], pl, rb0, mr0)
    best = min(table, key=lambda r: r["ms"])
    for rb in root_blocks:
        if rb != rb0:
            measure(best["enum_min_blocks"], best["lane_leaf_max"], best["planner"], rb, mr0)
    best = min(table, key=lambda r: r["ms"])
    for mr in merge_ratios:
        if mr != mr0:
            measure(best["enum_min_blocks"], best["lane_leaf_max"], best["planner"], best["root_block_min"], mr)
    best = min(table, key=lambda r: r["ms"])
    dg.set_tuning(best["enum_min_blocks"], best["lane_leaf_max"], best["planner"], best["root_block_min"],
                  merge_ratio=best["merge_ratio"])
    return best, table
