#!/usr/bin/env python
"""Benchmark of the matching and counting path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2|c0]

Workload (default ``c2``): the config-1 data graph (seeded Chung-Lu, N=3.77M,
M=16.5M, degree exponent 2.1, 20 labels Zipf(1.2)) resident in HBM, and the
config-2 mixed batch: the first 1,000 random-walk queries in seed order, sizes
uniform in 4..32, none screened out.  One step = every query of the batch
through candidate-space construction, planning and exact counting, with a
per-query cap on the enumeration (``--query-cap`` seconds of GPU time, the time
the query would run alone on the GPU).  Each query ends the step with one
status:

* ok       — the exact uint64 count;
* overflow — the count is shown to be at least 2^64 (a lower bound formed on
             the device proves it; a uint64 count cannot hold it);
* timeout  — the cap ran out first (recorded, never dropped).

``value`` is the batched form (one launch per CFL phase for the whole batch,
one persistent enumeration kernel over every (query, root block)):
queries of the batch per second, timeouts included at their cap.  The plain
form (one query per launch sequence, same cap) and the batched form with
learned plans are timed too.  Every step checks every exact count against the
reference's counts where the reference finished (tests/golden/c2_batch.json)
and against every other step and form.

Multi-GPU: the path shards by query; rank r takes every N-th query of the
batch, with no collective on the data path ("scaling": "weak" in the sense
that each rank holds its own copy of the graph; the batch is split); the value
is the batch's queries / the slowest rank's step time.

``--impl reference`` times the reference's own CPU build (oracle/_ref/ref_count,
the ALL_LEVEL mode that gives exact counts) on the same batch: its input files
come from the host-only generator asdmatch_b200/bin/asdm_gen.out, and the
process never loads this library.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
GOLDEN_C2 = os.path.join(ROOT, "tests", "golden", "c2_batch.json")
REF_COUNT = os.path.join(ROOT, "oracle", "_ref", "ref_count")
GEN = os.path.join(ROOT, "asdmatch_b200", "bin", "asdm_gen.out")
TWO64 = 1 << 64
OK, OVERFLOW, TIMEOUT = 0, 5, 6
STATUS_NAME = {OK: "ok", OVERFLOW: "overflow", TIMEOUT: "timeout"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c0"])
    ap.add_argument("--query-cap", type=float, default=0.02,
                    help="GPU seconds of enumeration one query may use (its time alone on the GPU)")
    ap.add_argument("--ref-cap", type=float, default=10.0, help="seconds one reference process may run")
    ap.add_argument("--cpu-sample", type=int, default=0, help="queries in the CPU-baseline sample (0: the host's cores)")
    ap.add_argument("--queries", type=int, default=0, help="use only the first K queries (profiling runs)")
    ap.add_argument("--profile", action="store_true", help="timed steps only: no other forms, no CPU baseline")
    ap.add_argument("--no-c4", action="store_true", help="skip the config-1 and config-4 measurements")
    ap.add_argument("--no-tune", action="store_true", help="keep the default kernel knobs (profiling runs)")
    ap.add_argument("--enum-min-blocks", type=int, default=0,
                    help="resident blocks per SM the enumeration kernel is compiled for (0: the library default "
                         "or the tuner's choice; profiling runs)")
    ap.add_argument("--root-block-min", type=int, default=0,
                    help="fewest level-0/1 pairs per root task of short plans (0: the library default or the "
                         "tuner's choice; profiling runs)")
    ap.add_argument("--padded-cap-log2", type=int, default=0,
                    help="candidate-edge build: padded lists up to 2^K entries, counting then filling beyond "
                         "(0: the library default; profiling runs)")
    ap.add_argument("--merge-ratio", type=int, default=-1,
                    help="intersection merge/gallop length ratio before tuning (-1: the library default)")
    ap.add_argument("--estimator", default="", help="learned-estimator parameters (.npy); default: the trained "
                                                    "config-1 model shipped with the package, when present")
    ap.add_argument("--learned-max", type=int, default=0, help="largest prefix the estimator is asked about (0 = 6)")
    return ap.parse_args()


def load_specs():
    """asdmatch_b200/specs.py by path: plain data, no import of the package (whose
    __init__ loads the compiled library)."""
    spec = importlib.util.spec_from_file_location("asdm_specs", os.path.join(ROOT, "asdmatch_b200", "specs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_golden():
    if not os.path.exists(GOLDEN_C2):
        return {}
    with open(GOLDEN_C2) as fh:
        return {r["index"]: r for r in json.load(fh)["queries"]}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return d.get("hbm_gbs", 6650.0), "measured (MEASURED_PEAKS.json hbm_gbs)"
    return 6650.0, "fallback: 6.65 TB/s, an earlier copy measurement on B200 (no MEASURED_PEAKS.json)"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def max_over_ranks(x, world, device):
    """The slowest rank's value (every rank calls this at the same point)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def flush_l2(torch, dev):
    # a 256 MB write evicts the 126 MB L2 between timed steps
    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    buf.fill_(1.0)
    torch.cuda.synchronize(dev)
    del buf


def histogram(values):
    out = {}
    for v in values:
        out[v] = out.get(v, 0) + 1
    return dict(sorted(out.items()))


class Checker:
    """Every exact count of every step and form must equal the reference's
    count where the reference finished, and every other exact count of the same
    query; an overflow must not meet an exact count."""

    def __init__(self, golden, indices):
        self.golden = golden
        self.indices = indices          # batch position -> query index in the C2 batch
        self.seen = {}                  # query index -> exact count first seen
        self.overflow = set()
        self.confirmed = set()          # answered and equal to a reference count

    def check(self, what, counts, status, positions=None):
        for pos, (c, st) in enumerate(zip(counts, status)):
            i = self.indices[pos if positions is None else positions[pos]]
            g = self.golden.get(i)
            st = int(st)
            if st == OK:
                c = int(c)
                if g is not None and g.get("count") is not None and g["count"] != c:
                    raise SystemExit("%s: query %d counts %d, the reference %d" % (what, i, c, g["count"]))
                if i in self.overflow or self.seen.setdefault(i, c) != c:
                    raise SystemExit("%s: query %d counts %d, another run %s" % (
                        what, i, c, "overflow" if i in self.overflow else self.seen[i]))
                if g is not None and g.get("count") is not None:
                    self.confirmed.add(i)
            elif st == OVERFLOW:
                if (g is not None and g.get("count") is not None) or i in self.seen:
                    raise SystemExit("%s: query %d overflow, but an exact count exists" % (what, i))
                self.overflow.add(i)
            elif st != TIMEOUT:
                raise SystemExit("%s: query %d failed with status %d" % (what, i, st))


# ----------------------------------------------------------------------------- reference arm

def reference_inputs(specs, indices, workdir):
    """The data graph and the batch's queries as t/v/e files, written by the
    host-only generator (cached in workdir)."""
    os.makedirs(workdir, exist_ok=True)
    dpath = os.path.join(workdir, "data.graph")
    if not os.path.exists(dpath):
        subprocess.run([GEN, "graph"] + specs.generator_args(specs.C1) + [dpath + ".tmp"], check=True)
        os.replace(dpath + ".tmp", dpath)
    missing = [i for i in indices if not os.path.exists(os.path.join(workdir, "q%d.graph" % i))]
    if missing:
        lst = os.path.join(workdir, "gen_list.txt")
        with open(lst, "w") as fh:
            for i in missing:
                seed, size = specs.c2_seed_size(i)
                fh.write("%d %d 0 q%d.graph\n" % (size, seed, i))
        subprocess.run([GEN, "queries"] + specs.generator_args(specs.C1) + [lst, workdir], check=True)
    return dpath, [os.path.join(workdir, "q%d.graph" % i) for i in indices]


def run_reference_queries(dpath, qpaths, jobs, cap, outdir):
    """oracle/_ref/ref_count over the queries: the data graph is read once, each
    query runs in its own forked single-threaded process (at most `jobs` at a
    time, each killed after `cap` seconds).  Returns per query
    (status, count, execution_s, wall_s) and the harness's wall time."""
    os.makedirs(outdir, exist_ok=True)
    lst = os.path.join(outdir, "list.txt")
    with open(lst, "w") as fh:
        fh.write("\n".join(qpaths) + "\n")
    t0 = time.time()
    r = subprocess.run([REF_COUNT, "-d", dpath, "-Q", lst, "-O", outdir, "-T", str(cap), "-J", str(jobs)],
                       capture_output=True, text=True)
    wall = time.time() - t0
    res = [None] * len(qpaths)
    for line in r.stdout.splitlines():
        parts = line.split()
        if len(parts) < 4 or parts[0] != "Q":
            continue
        k = int(parts[1])
        st = parts[2]
        qwall = float(parts[-1])
        count = execs = None
        if st == "ok":
            with open(os.path.join(outdir, "q%d.out" % k)) as fh:
                for l in fh:
                    if l.startswith("Number of matches:"):
                        count = int(l.split(":")[1])
                    elif l.startswith("Execution Time:"):
                        execs = float(l.split(":")[1])
        res[k] = (st, count, execs, qwall)
    # a query the harness never reported (it died) counts as a capped failure
    res = [r if r is not None else ("missing", None, None, float(cap)) for r in res]
    return res, wall


def graph_load_seconds(dpath):
    """Wall time of the reference reading the data graph (one process, no query)."""
    t0 = time.time()
    subprocess.run([REF_COUNT, "-d", dpath, "-Q", os.devnull, "-O", tempfile.gettempdir()], capture_output=True)
    return time.time() - t0


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    if not os.path.exists(REF_COUNT) or not os.path.exists(GEN):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref/ref_count) or the "
                                                              "host-only generator (asdm_gen.out) is not built"}))
        return
    specs = load_specs()
    golden = load_golden()
    per_step = cores
    total = (args.warmup + args.steps) * per_step
    indices = [i % specs.C2_QUERIES for i in range(total)]
    workdir = os.environ.get("ASDM_BENCH_CACHE") or os.path.join(tempfile.gettempdir(), "asdm_c2_inputs")
    dpath, qpaths = reference_inputs(specs, sorted(set(indices)), workdir)
    qmap = dict(zip(sorted(set(indices)), qpaths))
    outdir = tempfile.mkdtemp(prefix="asdm_ref_out_")
    res, harness_wall = run_reference_queries(dpath, [qmap[i] for i in indices], cores, args.ref_cap, outdir)
    load_s = graph_load_seconds(dpath)
    timed = res[args.warmup * per_step:]
    walls = [r[3] for r in timed]
    execs = [r[2] for r in timed if r[2] is not None]
    answered = [(indices[args.warmup * per_step + k], r[1]) for k, r in enumerate(timed) if r[0] == "ok"]
    wrong = [i for i, c in answered if golden.get(i, {}).get("count") not in (None, c)]
    stats = histogram(r[0] for r in timed)
    # throughput of `cores` concurrent processes: each query costs its own wall time (capped)
    value = cores / statistics.mean(walls)
    ms_per_step = 1000.0 * statistics.mean(walls) * per_step / cores
    sizes = [specs.c2_seed_size(i)[1] for i in indices[args.warmup * per_step:]]
    cfg = {"workload": "c2: config-1 graph (Chung-Lu N=3.77M M=16.5M gamma=2.1, 20 labels Zipf(1.2)); the first 1,000 "
                       "random-walk queries in seed order, sizes uniform 4..32, none screened out",
           "graph": specs.C1, "queries": specs.C2_QUERIES, "sample_query_sizes": histogram(sizes),
           "per_query_cap_s": args.ref_cap}
    line = {"metric": "exact-count queries/sec", "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint32 ids / uint64 counts",
            "data": "synthetic (seeded generators; no dataset download)", "config": cfg, "impl": "reference",
            "cpu_baseline": {
                "value": value, "unit": "queries/s", "cores": cores, "kind": "reference",
                "sample": "queries %d..%d of the batch after %d warm-up queries, %d per step, %d concurrent "
                          "single-threaded reference processes (ALL_LEVEL build) forked after one graph load "
                          "(%.1f s, not counted), each capped at %.0f s; statuses %s; the reference's own summed "
                          "'Execution Time' %.1f s over %d finished queries, wall %.1f s over all; counts that "
                          "differ from the reference goldens: %d" % (
                              indices[args.warmup * per_step], indices[-1], args.warmup * per_step, per_step, cores,
                              load_s, args.ref_cap, stats, sum(execs), len(execs), sum(walls), len(wrong))},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ----------------------------------------------------------------------------- our arm

def shard(items, rank, world):
    """The batch split by query: rank r takes every world-th query from r on."""
    return list(items)[rank::world]


def setup_workload(name, rank, world, limit):
    import asdmatch_b200 as A
    from asdmatch_b200 import workloads as W
    if name == "c0":
        g = W.graph(W.C0)
        qs = W.queries(g, 8, 200, W.C0_QUERY_SEED + 800)
        with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as fh:
            golden = {r["index"]: r for r in json.load(fh)["sets"]["c0"]}
        indices = list(range(len(qs)))
        cfg = {"workload": "c0: Chung-Lu N=3112 M=12519 gamma=2.5 71 labels Zipf(1.0); 200 random-walk queries of 8 "
                           "vertices", "graph": W.C0}
    else:
        g = W.graph(W.C1)
        n = limit or W.C2_QUERIES
        indices = list(range(n))
        qs = W.c2_batch(g, n)
        golden = load_golden()
        sizes = [W.c2_seed_size(i)[1] for i in indices]
        cfg = {"workload": "c2: config-1 graph (Chung-Lu N=3.77M M=16.5M gamma=2.1, 20 labels Zipf(1.2)) resident "
                           "in HBM; the first %d random-walk queries in seed order, sizes uniform 4..32, none "
                           "screened out" % n,
               "graph": W.C1, "queries": n, "query_sizes": histogram(sizes),
               "query_cycle_rank": histogram(q.m2 // 2 - q.n + 1 for q in qs)}
    if world > 1:
        qs, indices = shard(qs, rank, world), shard(indices, rank, world)
    return A, W, g, qs, indices, golden, cfg


def cpu_baseline(dpath, qpaths, cap):
    """The reference's own CPU path (oracle/_ref/ref_count) on a bounded sample of
    the batch, all host cores, one forked process per query."""
    cores = os.cpu_count() or 1
    if not os.path.exists(REF_COUNT):
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "unavailable",
                "sample": "oracle/_ref is not built"}
    res, wall = run_reference_queries(dpath, qpaths, cores, cap, tempfile.mkdtemp(prefix="asdm_cpu_"))
    walls = [r[3] for r in res]
    execs = [r[2] for r in res if r[2] is not None]
    return {"value": cores / statistics.mean(walls), "unit": "queries/s", "cores": cores, "kind": "reference",
            "sample": "the batch's first %d queries, %d concurrent single-threaded reference processes (ALL_LEVEL "
                      "build) forked after one graph load, each capped at %.0f s; statuses %s; summed 'Execution "
                      "Time' %.1f s over %d finished" % (len(qpaths), cores, cap, histogram(r[0] for r in res),
                                                         sum(execs), len(execs))}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    sys.path.insert(0, ROOT)
    import numpy as np
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    A, W, g, qs, indices, golden, cfg = setup_workload(args.workload, rank, world, args.queries)
    dg = A.DeviceGraph(g)
    if args.padded_cap_log2 or args.enum_min_blocks or args.root_block_min or args.merge_ratio >= 0:
        t = dg.tuning()
        dg.set_tuning(args.enum_min_blocks or t["enum_min_blocks"], t["lane_leaf_max"],
                      root_block_min=args.root_block_min or t["root_block_min"],
                      padded_cap_log2=args.padded_cap_log2 or t["padded_cap_log2"],
                      merge_ratio=args.merge_ratio if args.merge_ratio >= 0 else t["merge_ratio"])
    stream = torch.cuda.ExternalStream(dg.stream(), device=dev)
    Q = len(qs)
    Qall = Q * world if world > 1 else Q
    cap = args.query_cap
    checker = Checker(golden, indices)
    packed = A.BatchInput(qs)

    def batched_step(estimator=None, batch=packed, check=True, what="batched"):
        st = A.run_batch_ex(dg, batch, estimator=estimator, learned_max_subset=args.learned_max,
                            query_time_limit_s=cap)
        if check:
            checker.check(what, batch.counts, batch.status)
        return {"kernel_ms": st.kernel_ms, "list_bytes": st.list_bytes, "cs_ms": st.build_ms,
                "cs_bytes": st.build_bytes, "matches": int(batch.counts[batch.status == OK].sum(dtype=np.uint64)),
                "inter": st.intersections, "busy_warp_ms": st.busy_warp_ms, "idle_warp_ms": st.idle_warp_ms,
                "tasks": st.tasks,
                "status": histogram(int(x) for x in batch.status)}

    def plain_step(positions=None):
        """The plain form: one query per launch sequence (candidate space, sampling
        estimates, plan, count), same cap; over the batch positions given (all)."""
        positions = list(range(Q)) if positions is None else positions
        counts = np.zeros(len(positions), np.uint64)
        status = np.zeros(len(positions), np.int32)
        agg = {"kernel_ms": 0.0, "list_bytes": 0, "cs_ms": 0.0, "cs_bytes": 0, "inter": 0}
        for k, q in enumerate(qs[p] for p in positions):
            cs = A.CandidateSpace(dg, q)
            b, ms_ = cs.build_stats()
            agg["cs_bytes"] += b
            agg["cs_ms"] += ms_
            if cs.nonempty:
                try:
                    plan = A.Plan(cs, card=A.Card.sample(cs, seed=k))
                    r = A.adaptive_share_join(cs, plan, time_limit_s=cap)
                    counts[k] = r.count
                    agg["kernel_ms"] += r.kernel_ms
                    agg["list_bytes"] += r.list_bytes
                    agg["inter"] += r.intersections
                except A.AsdmError as e:
                    if e.code not in (OVERFLOW, TIMEOUT):
                        raise
                    status[k] = e.code
            cs.close()
        checker.check("plain", counts, status, positions)
        agg["matches"] = int(counts[status == OK].sum(dtype=np.uint64))
        agg["status"] = histogram(int(x) for x in status)
        return agg

    def timed(step_fn, steps):
        times, agg = [], None
        for _ in range(steps):
            flush_l2(torch, dev)
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = step_fn()
            e1.record(stream)
            e1.synchronize()
            torch.cuda.synchronize(dev)
            times.append(e0.elapsed_time(e1))
            agg = st if agg is None else {k: (agg[k] + st[k] if k != "status" else st[k]) for k in agg}
        return max_over_ranks(statistics.mean(times), world, dev), agg

    # warm-up (first step also picks the queries the tuner times: those counted exactly)
    first = batched_step()
    first_status = packed.status.tolist()
    exact = [q for q, s in zip(qs, first_status) if s == OK]
    if args.no_tune or not exact:
        tune_best, tune_table = dg.tuning(), []
    else:
        tune_batch = A.BatchInput(exact)
        tune_best, tune_table = A.autotune(dg, tune_batch, reps=1,
                                           run=lambda d, b: A.run_batch_ex(d, b, query_time_limit_s=cap))
    for _ in range(max(0, args.warmup - 1)):
        batched_step()
    sampler = ClockSampler(local)
    launches0 = A.kernel_launches()
    sampler.start()
    ms, agg = timed(batched_step, args.steps)
    clocks = sampler.stop()
    launches = A.kernel_launches() - launches0
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms, "queries": Q, "status": agg["status"],
                              "enum_kernel_ms_per_step": agg["kernel_ms"] / args.steps,
                              "cs_build_ms_per_step": agg["cs_ms"] / args.steps,
                              "enum_algorithmic_bytes_per_step": agg["list_bytes"] / args.steps,
                              "enum_busy_warp_ms_per_step": agg["busy_warp_ms"] / args.steps,
                              "enum_idle_warp_ms_per_step": agg["idle_warp_ms"] / args.steps,
                              "enum_root_tasks_per_step": agg["tasks"] / args.steps,
                              "cs_algorithmic_bytes_per_step": agg["cs_bytes"] / args.steps,
                              "launches": launches // args.steps,
                              "tuning": dg.tuning(), "autotune_table": tune_table}))
        if world > 1:
            dist.destroy_process_group()
        return
    # the plain form, for the batched / plain ratio
    plain_step()
    plain_ms, plain_agg = timed(plain_step, args.steps)
    # batched with learned plans
    est = None
    est_path = args.estimator
    if not est_path:
        from asdmatch_b200 import estimator as E
        est_path = E.DEFAULT_PARAMS if os.path.exists(E.DEFAULT_PARAMS) else ""
    learned = None
    if est_path:
        est = A.Estimator(A.EST_FEATURES, 0)
        est.set_params(np.load(est_path))
        batched_step(estimator=est, what="learned")
        learned_ms, learned_agg = timed(lambda: batched_step(estimator=est, what="learned"), args.steps)
        learned = {"queries_per_s": Qall / (learned_ms / 1e3), "ms_per_step": learned_ms,
                   "status": {STATUS_NAME.get(k, k): v for k, v in learned_agg["status"].items()},
                   "enum_kernel_ms_per_step": learned_agg["kernel_ms"] / args.steps,
                   "cs_build_ms_per_step": learned_agg["cs_ms"] / args.steps,
                   "over_plain": plain_ms / learned_ms, "over_cost_model_batched": ms / learned_ms,
                   "estimator": os.path.relpath(est_path, ROOT) if est_path.startswith(ROOT) else est_path,
                   "learned_max_subset": args.learned_max or 6,
                   "what": "asdm_run_batch_ex with the learned estimator: candidate spaces, learned plans (one "
                           "forward pass per planner step for the whole group), one persistent launch; planning is "
                           "inside the timed region"}
    # the same forms on the queries the first step decided (exact count or proven overflow): timeouts,
    # which cost their cap in every form, left out
    decided_pos = [p for p, s in enumerate(first_status) if s in (OK, OVERFLOW)]
    decided = None
    if decided_pos:
        dbatch = A.BatchInput([qs[p] for p in decided_pos])

        def decided_batched(estimator=None, what="batched-decided"):
            st = A.run_batch_ex(dg, dbatch, estimator=estimator, learned_max_subset=args.learned_max,
                                query_time_limit_s=cap)
            checker.check(what, dbatch.counts, dbatch.status, decided_pos)
            return {"status": histogram(int(x) for x in dbatch.status)}

        decided_batched()
        d_ms, d_agg = timed(decided_batched, args.steps)
        d_plain_ms, _ = timed(lambda: plain_step(decided_pos), args.steps)
        decided = {"queries": len(decided_pos), "batched_ms": d_ms, "plain_ms": d_plain_ms,
                   "batched_queries_per_s": world * len(decided_pos) / (d_ms / 1e3),
                   "batched_over_plain": d_plain_ms / d_ms,
                   "status": {STATUS_NAME.get(k, k): v for k, v in d_agg["status"].items()}}
        if est is not None:
            d_learned_ms, _ = timed(lambda: decided_batched(est, "learned-decided"), args.steps)
            decided.update(learned_ms=d_learned_ms, learned_over_plain=d_plain_ms / d_learned_ms)
    # end to end through the C ABI (asdm_run_batch_ex) from host arrays, same cold-L2 protocol
    e2e_times = []
    h2d = packed.nbytes()
    d2h = Q * (8 + 4)
    for _ in range(args.steps):
        flush_l2(torch, dev)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        A.run_batch_ex(dg, packed, query_time_limit_s=cap)
        e2e_times.append(time.perf_counter() - t0)
        checker.check("e2e", packed.counts, packed.status)
    e2e_s = max_over_ranks(statistics.mean(e2e_times), world, dev)
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    peak, peak_kind = measured_peaks()
    steps = args.steps
    enum_ms, cs_ms = agg["kernel_ms"] / steps, agg["cs_ms"] / steps
    bytes_ = agg["list_bytes"] / steps
    achieved = bytes_ / (enum_ms * 1e-3) / 1e9 if enum_ms > 0 else 0.0
    cs_bytes = agg["cs_bytes"] / steps
    cs_achieved = cs_bytes / (cs_ms * 1e-3) / 1e9 if cs_ms > 0 else 0.0
    traffic = traffic_cs = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        # DRAM bytes per algorithmic byte from an ncu capture of a smaller case of the same workload,
        # scaled to this step's algorithmic bytes
        with open(tp) as fh:
            t = json.load(fh).get(args.workload) or {}

        def scaled(k, alg):
            e = t.get(k)
            ok = isinstance(e, dict) and e.get("algorithmic_bytes") and e.get("dram_bytes") is not None
            return round(e["dram_bytes"] / e["algorithmic_bytes"] * alg) if ok else None
        traffic, traffic_cs = scaled("enum_batch_kernel", bytes_), scaled("k1_k3", cs_bytes)
    status = {STATUS_NAME.get(k, k): v for k, v in agg["status"].items()}
    n_decided = status.get("ok", 0) + status.get("overflow", 0)
    line = {
        "metric": "exact-count queries/sec",
        "value": Qall / (ms / 1e3),
        "unit": "queries/s",
        "n_gpus": world,
        "steps": steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "uint32 ids / uint64 counts",
        "data": "synthetic (seeded generators; no dataset download)",
        "config": dict(cfg, l2="flushed (256 MB write) before every timed step",
                       per_query_cap_s=cap,
                       per_query_cap="GPU time of enumeration a query may use: its warp-time over all resident "
                                     "warps, i.e. the time it would run alone on the GPU (timeouts are counted "
                                     "at the cap and reported, never dropped)",
                       status_per_step=status,
                       decided_queries_per_s=world * n_decided / (ms / 1e3),
                       exact_counts_confirmed_by_reference=len(checker.confirmed),
                       form="batched: asdm_run_batch_ex (one launch per CFL phase for the group, tree program, "
                            "overflow lower bounds, one persistent enumeration kernel over all (query, root task) "
                            "pairs); planner: candidate-size cost model, " +
                            ("exhaustive prefix search" if tune_best.get("planner", 0) == A.PLANNER_DP else "greedy"),
                       matches_per_step=agg["matches"] // steps,
                       matches_per_s=world * (agg["matches"] // steps) / (ms / 1e3),
                       intersections_per_step=agg["inter"] // steps,
                       enum_kernel_ms_per_step=enum_ms, cs_build_ms_per_step=cs_ms,
                       plain_form={"queries_per_s": Qall / (plain_ms / 1e3), "ms_per_step": plain_ms,
                                   "status": {STATUS_NAME.get(k, k): v for k, v in plain_agg["status"].items()},
                                   "enum_kernel_ms_per_step": plain_agg["kernel_ms"] / steps,
                                   "cs_build_ms_per_step": plain_agg["cs_ms"] / steps,
                                   "what": "one query per launch sequence (asdm_candidate_space, asdm_card_sample: "
                                           "the sampling estimator, asdm_plan_create_card, asdm_run_plan with the "
                                           "same cap as a time limit)"},
                       batched_over_plain=plain_ms / ms,
                       decided_subset=decided,
                       cs_build_roofline={"kernels": "K1-K3 (k1_filter, k2_pull, compaction, k3_bound/flat/pack)",
                                          "bound": "hbm", "achieved": cs_achieved, "peak": peak, "unit": "GB/s",
                                          "frac": cs_achieved / peak, "algorithmic_bytes_per_step": cs_bytes,
                                          "device_ms_per_step": cs_ms, "traffic": traffic_cs},
                       batched_learned=learned,
                       autotune={"chosen": tune_best, "table": tune_table,
                                 "tuned_on": "%d queries counted exactly in the first warm-up step" % len(exact)},
                       first_step_status={STATUS_NAME.get(k, k): v for k, v in first["status"].items()}),
        "roofline": {"kernel": "enum_batch_kernel (K4-K8 warp DFS, batched)", "bound": "hbm", "achieved": achieved,
                     "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": bytes_, "device_ms_per_step": enum_ms, "traffic": traffic},
        "e2e": {"value": Qall / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "via": "asdm_run_batch_ex (C ABI) from host arrays, wall clock, L2 flushed before each step"},
        "gpu_launches": launches // steps,
        "clocks": clocks,
    }
    if world == 1 and not args.no_c4 and args.workload == "c2":
        line["config"]["config1"] = measure_c1(A, W, g, dg, torch, dev, args.steps, cap)
        line["config"]["local_counting_c4"] = measure_c4(A, W, torch, dev, args.steps, cap)
    if world == 1 and args.workload == "c2":
        tmp = tempfile.mkdtemp(prefix="asdm_cpu_")
        n = args.cpu_sample or (os.cpu_count() or 1)
        dpath, qpaths = W.write_workload(tmp, g, qs[:n])
        line["cpu_baseline"] = cpu_baseline(dpath, qpaths, args.ref_cap)
    print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def csv_sha256(mat):
    """SHA-256 of a local-count matrix written the way the reference writes its
    CSV (main.cpp:135-146): one row per data vertex, ',' between columns."""
    import hashlib
    h = hashlib.sha256()
    for r0 in range(0, mat.shape[0], 65536):
        block = mat[r0:r0 + 65536]
        h.update(("\n".join(",".join(map(str, row)) for row in block.tolist()) + "\n").encode())
    return h.hexdigest()


def measure_c1(A, W, g, dg, torch, dev, steps, cap):
    """Config 1: 100 queries each of 12 and 16 vertices (half dense, half sparse)
    on the resident config-1 graph, batched with the per-query cap; per-query
    wall times from the plain form (one query per launch sequence)."""
    import numpy as np
    batch = W.c1_batch(g)
    qs = [q for _, _, _, q in batch]
    classes = ["%d-%s" % (size, "dense" if d == W.DENSE else "sparse") for size, d, _, _ in batch]
    stream = torch.cuda.ExternalStream(dg.stream(), device=dev)
    b = A.BatchInput(qs)
    A.run_batch_ex(dg, b, query_time_limit_s=cap)  # warm
    times = []
    for _ in range(steps):
        flush_l2(torch, dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        A.run_batch_ex(dg, b, query_time_limit_s=cap)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    by_class = {}
    for c, st in zip(classes, b.status.tolist()):
        by_class.setdefault(c, {})
        k = STATUS_NAME.get(st, st)
        by_class[c][k] = by_class[c].get(k, 0) + 1
    walls = []
    for q, st in zip(qs, b.status.tolist()):
        t0 = time.perf_counter()
        cs = A.CandidateSpace(dg, q)
        try:
            if cs.nonempty:
                A.adaptive_share_join(cs, time_limit_s=cap)
        except A.AsdmError as e:
            if e.code not in (OVERFLOW, TIMEOUT):
                raise
        cs.close()
        walls.append(time.perf_counter() - t0)
    walls.sort()
    ms = statistics.mean(times)
    return {"workload": "config 1: config-1 graph; 100 random-walk queries each of 12 and 16 vertices, half dense "
                        "(average degree >= 3), half sparse; per-query cap %.3g s of GPU time (the reference's is "
                        "300 s of CPU)" % cap,
            "queries_per_s": len(qs) / (ms / 1e3), "ms_per_step": ms, "status_by_class": by_class,
            "plain_per_query_wall_s": {"median": walls[len(walls) // 2], "p90": walls[int(0.9 * len(walls))],
                                       "max": walls[-1]},
            "via": "asdm_run_batch_ex (batched); per-query walls: asdm_candidate_space + asdm_run_plan with the cap "
                   "as time limit"}


def measure_c4(A, W, torch, dev, steps, cap):
    """Config 4: 50 random-walk queries of 10 vertices on the 1M/10M graph,
    batched LOCAL_COUNT with the per-query cap; every finished query's
    |Vg| x |Vq| matrix sums to its count in every column, and its CSV digest
    equals the reference's where the reference finished
    (tests/golden/c4_batch.json)."""
    import numpy as np
    g = W.graph(W.C4)
    qs = W.c4_batch(g)
    golden = {}
    gp = os.path.join(ROOT, "tests", "golden", "c4_batch.json")
    if os.path.exists(gp):
        with open(gp) as fh:
            golden = {r["index"]: r for r in json.load(fh)["queries"]}
    dg = A.DeviceGraph(g)
    stream = torch.cuda.ExternalStream(dg.stream(), device=dev)
    counts, status, mats, _ = A.run_batch_local_ex(dg, qs, query_time_limit_s=cap)  # warm
    first = (counts.copy(), status.copy())
    confirmed = 0
    for k, (c, st, m) in enumerate(zip(counts.tolist(), status.tolist(), mats)):
        r = golden.get(k)
        if st == OK:
            if any(int(x) != c for x in m.sum(axis=0, dtype=np.uint64)):
                raise SystemExit("config-4 query %d: local counts do not sum to the count" % k)
            if r is not None and r.get("count") is not None:
                if r["count"] != c or r.get("csv_sha256") != csv_sha256(m):
                    raise SystemExit("config-4 query %d differs from the reference" % k)
                confirmed += 1
        elif st not in (OVERFLOW, TIMEOUT):
            raise SystemExit("config-4 query %d failed with status %d" % (k, st))
        elif r is not None and r.get("count") is not None and st == OVERFLOW:
            raise SystemExit("config-4 query %d: overflow, but the reference finished" % k)
    times = []
    for _ in range(steps):
        flush_l2(torch, dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        counts, status, mats, _ = A.run_batch_local_ex(dg, qs, query_time_limit_s=cap)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        ok = (status == OK) & (first[1] == OK)
        if not np.array_equal(counts[ok], first[0][ok]):
            raise SystemExit("config-4 counts changed between steps")
    ms = statistics.mean(times)
    dg.close()
    return {"workload": "config 4: Chung-Lu N=1.0M M=10M gamma=2.3, 32 labels Zipf(1.0); 50 random-walk queries of "
                        "10 vertices, LOCAL_COUNT; per-query cap %.3g s of GPU time" % cap,
            "queries_per_s": len(qs) / (ms / 1e3), "ms_per_step": ms,
            "status": {STATUS_NAME.get(k, k): v for k, v in histogram(int(x) for x in status).items()},
            "csv_equal_to_reference": confirmed,
            "local_count_bytes_per_step": 8 * g.n * sum(q.n for q, st in zip(qs, status.tolist()) if st == OK),
            "via": "asdm_run_batch_ex with local-count matrices (|Vg| x |Vq| uint64, copied to host every step)"}


if __name__ == "__main__":
    main()
