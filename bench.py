#!/usr/bin/env python
"""Benchmark of the matching and counting path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload c2|c0]

Workload (default ``c2``): the config-1 data graph (seeded Chung-Lu, N=3.77M,
M=16.5M, degree exponent 2.1, 20 labels Zipf(1.2)) resident in HBM, and the
config-2 mixed batch of random-walk queries with sizes uniform in 4..32,
screened to the queries whose exact count is at most 10^9 (the screen and its
exact counts are in asdmatch_b200/c2_screened.json).  One step = every query
of the batch through candidate-space construction, planning and exact
counting.  ``value`` is the batched form (asdm_run_batch: one launch per CFL
phase for the whole batch, one persistent enumeration kernel over every
(query, root block)), with the kernel knobs picked by the autotuner before
timing; the plain form (one query per launch sequence) is timed too and
reported in ``config.plain_form``.  Every step's counts are checked against
the screened counts.

Multi-GPU: the path shards by query; every rank runs the whole batch on its
own GPU with no collective on the data path ("scaling": "weak"); the value is
N x queries / the slowest rank's step time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c0"])
    ap.add_argument("--cpu-sample", type=int, default=1, help="queries in the CPU-baseline sample")
    ap.add_argument("--queries", type=int, default=0, help="use only the first K queries (profiling runs)")
    ap.add_argument("--profile", action="store_true", help="timed steps only: no e2e pass, no CPU baseline")
    ap.add_argument("--no-c4", action="store_true", help="skip the config-4 local-counting measurement")
    ap.add_argument("--no-tune", action="store_true", help="keep the default kernel knobs (profiling runs)")
    ap.add_argument("--estimator", default="", help="learned-estimator parameters (.npy); default: the trained "
                                                    "config-1 model shipped with the package, when present")
    ap.add_argument("--learned-max", type=int, default=0, help="largest prefix the estimator is asked about (0 = 6)")
    return ap.parse_args()


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


def cpu_baseline(dpath, qpaths, want_counts, timeout_s=120):
    """The reference's own CPU path (oracle/_ref, ALL_LEVEL build), one process per
    query as the reference runs, else the oracle port; returns the JSON object."""
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_count")
    port = os.path.join(ROOT, "oracle", "_build", "asdm_oracle")
    exe, kind = (ref, "reference") if os.path.exists(ref) else (port, "port")
    if not os.path.exists(exe):
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "unavailable",
                "sample": "neither oracle/_ref nor oracle/_build is built"}
    done, t0 = 0, time.time()
    ok = True
    for qp, want in zip(qpaths, want_counts):
        try:
            r = subprocess.run([exe, "-q", qp, "-d", dpath], capture_output=True, text=True, timeout=timeout_s)
        except subprocess.TimeoutExpired:
            break
        got = [int(l.split(":")[1]) for l in r.stdout.splitlines() if l.startswith("Number of matches:")]
        ok &= bool(got) and got[0] == want
        done += 1
    dt = time.time() - t0
    return {"value": (done / dt) if done else 0.0, "unit": "queries/s", "cores": 1, "kind": kind,
            "sample": "%d of the batch's queries, one single-threaded process per query (graph load, CFL filter, "
                      "FHD planning, ALL_LEVEL join), %.1f s wall, counts %s" % (done, dt, "match" if ok else "DIFFER")}


def measure_c4(A, W, torch, dev, steps):
    """Config 4: the screened 8-vertex queries on the 1M/10M graph, batched LOCAL_COUNT
    (asdm_run_batch_local); checked every step (counts, and every local-count column sums
    to the count)."""
    import numpy as np
    g = W.graph(W.C4)
    sc = W.load_c4_screen()
    qs = W.c4_queries(g, sc)
    want = [r["count"] for r in sc["queries"]]
    dg = A.DeviceGraph(g)
    stream = torch.cuda.ExternalStream(dg.stream(), device=dev)
    A.run_batch_local(dg, qs)  # warm
    times = []
    for _ in range(steps):
        flush_l2(torch, dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        counts, status, mats = A.run_batch_local(dg, qs)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        if counts.tolist() != want or status.any():
            raise SystemExit("config-4 counts differ from the screened counts")
        for c, m in zip(want, mats):
            if any(int(x) != c for x in m.sum(axis=0, dtype=np.uint64)):
                raise SystemExit("config-4 local counts do not sum to the count")
    ms = statistics.mean(times)
    dg.close()
    return {"workload": "c4-screened: Chung-Lu N=1.0M M=10M gamma=2.3, 32 labels Zipf(1.0); %d random-walk queries "
                        "of %d vertices with <= 1e9 matches (%d of %d candidates; no 10-vertex query qualified)"
                        % (len(qs), sc["size"], len(qs), sc["candidates"]),
            "queries_per_s": len(qs) / (ms / 1e3), "ms_per_step": ms, "matches_per_step": int(sum(want)),
            "local_count_bytes_per_step": 8 * g.n * sum(q.n for q in qs),
            "via": "asdm_run_batch_local, |Vg| x |Vq| uint64 matrices copied to host every step"}


def setup_workload(name):
    import asdmatch_b200 as A
    from asdmatch_b200 import workloads as W
    if name == "c0":
        g = W.graph(W.C0)
        qs = W.queries(g, 8, 200, W.C0_QUERY_SEED + 800)
        with open(os.path.join(ROOT, "tests", "golden", "golden.json")) as fh:
            counts = [r["count"] for r in json.load(fh)["sets"]["c0"]]
        cfg = {"workload": "c0: Chung-Lu N=3112 M=12519 gamma=2.5 71 labels Zipf(1.0); 200 random-walk queries of 8 vertices",
               "graph": W.C0}
        return A, W, g, qs, counts, cfg
    g = W.graph(W.C1)
    sc = W.load_c2_screen()
    qs = W.c2_queries(g, sc)
    counts = [r["count"] for r in sc["queries"]]
    sizes = [r["size"] for r in sc["queries"]]
    cfg = {"workload": "c2-screened: config-1 graph (Chung-Lu N=3.77M M=16.5M gamma=2.1, 20 labels Zipf(1.2)) "
                       "resident in HBM; %d random-walk queries, sizes uniform 4..32 (mixed density), kept when the "
                       "exact count <= 1e9 (%d of %d candidates)" % (len(qs), len(qs), sc["candidates"]),
           "graph": W.C1, "queries": len(qs), "query_sizes": [min(sizes), max(sizes)],
           "count_limit": sc["count_limit"]}
    return A, W, g, qs, counts, cfg


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    import asdmatch_b200 as A  # generators only
    A_, W, g, qs, counts, cfg = setup_workload(args.workload)
    ref = os.path.join(ROOT, "oracle", "_ref", "ref_count")
    port = os.path.join(ROOT, "oracle", "_build", "asdm_oracle")
    exe, kind = (ref, "reference") if os.path.exists(ref) else (port, "port")
    if not os.path.exists(exe):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build (oracle/_ref) and oracle port missing"}))
        return
    cores = os.cpu_count() or 1
    tmp = tempfile.mkdtemp(prefix="asdm_ref_")
    dpath = os.path.join(tmp, "data.graph")
    g.write(dpath)
    qpaths = []
    for i, q in enumerate(qs):
        p = os.path.join(tmp, "q%d.graph" % i)
        q.write(p)
        qpaths.append(p)

    def step(k):
        # one bounded sample per step: `cores` queries in parallel, one reference process each
        idx = [(k * cores + j) % len(qs) for j in range(cores)]
        t0 = time.time()
        procs = [subprocess.Popen([exe, "-q", qpaths[i], "-d", dpath], stdout=subprocess.PIPE, text=True) for i in idx]
        good = 0
        for i, p in zip(idx, procs):
            out, _ = p.communicate()
            got = [int(l.split(":")[1]) for l in out.splitlines() if l.startswith("Number of matches:")]
            good += bool(got) and got[0] == counts[i]
        return time.time() - t0, good, len(idx)

    for k in range(args.warmup):
        step(k)
    t_total, good, n = 0.0, 0, 0
    for k in range(args.steps):
        dt, gd, nn = step(args.warmup + k)
        t_total += dt
        good += gd
        n += nn
    value = n / t_total
    line = {"metric": "exact-count queries/sec", "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * t_total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "uint32/uint64",
            "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": kind,
                             "sample": "%d queries per step on %d cores (one single-threaded reference process per "
                                       "query), counts correct %d/%d" % (cores, cores, good, n)},
            "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)
    A, W, g, qs, counts, cfg = setup_workload(args.workload)
    if args.queries:
        qs, counts = qs[:args.queries], counts[:args.queries]
        cfg = dict(cfg, queries=len(qs), subset="first %d queries" % len(qs))
    dg = A.DeviceGraph(g)
    stream = torch.cuda.ExternalStream(dg.stream(), device=dev)
    Q = len(qs)

    def plain_step():
        """The plain form: one query per launch sequence (candidate space, plan, count)."""
        stats = {"kernel_ms": 0.0, "list_bytes": 0, "cs_ms": 0.0, "cs_bytes": 0, "matches": 0, "inter": 0}
        for q, want in zip(qs, counts):
            cs = A.CandidateSpace(dg, q)
            b, ms_ = cs.build_stats()
            stats["cs_bytes"] += b
            stats["cs_ms"] += ms_
            if cs.nonempty:
                r = A.adaptive_share_join(cs)
                stats["kernel_ms"] += r.kernel_ms
                stats["list_bytes"] += r.list_bytes
                stats["inter"] += r.intersections
                got = r.count
            else:
                got = 0
            cs.close()
            if got != want:
                raise SystemExit("count mismatch: %d != %d" % (got, want))
            stats["matches"] += got
        return stats

    packed = A.BatchInput(qs)
    if args.no_tune:
        tune_best, tune_table = dg.tuning(), []
    else:
        tune_best, tune_table = A.autotune(dg, packed)  # untimed: picks the kernel knobs on this batch

    def batched_step():
        """The batched form: the whole batch through asdm_run_batch."""
        st = A.run_batch_packed(dg, packed)
        if packed.counts.tolist() != counts or packed.status.any():
            raise SystemExit("batched counts differ from the screened counts")
        return {"kernel_ms": st.kernel_ms, "list_bytes": st.list_bytes, "cs_ms": st.build_ms,
                "cs_bytes": st.build_bytes, "matches": st.count, "inter": st.intersections}

    est = None
    est_path = args.estimator
    if not est_path:
        from asdmatch_b200 import estimator as E
        est_path = E.DEFAULT_PARAMS if os.path.exists(E.DEFAULT_PARAMS) else ""
    if est_path:
        est = A.Estimator(A.EST_FEATURES, 0)
        est.set_params(np.load(est_path))

    def learned_step():
        """Batched + learned: asdm_run_batch_ex with the estimator planning every query."""
        st = A.run_batch_ex(dg, packed, estimator=est, learned_max_subset=args.learned_max)
        if packed.counts.tolist() != counts or packed.status.any():
            raise SystemExit("learned-plan counts differ from the screened counts")
        return {"kernel_ms": st.kernel_ms, "list_bytes": st.list_bytes, "cs_ms": st.build_ms,
                "cs_bytes": st.build_bytes, "matches": st.count, "inter": st.intersections}

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
            agg = st if agg is None else {k: agg[k] + st[k] for k in agg}
        return max_over_ranks(statistics.mean(times), world, dev), agg

    for _ in range(args.warmup):
        batched_step()
    sampler = ClockSampler(local)
    launches0 = A.kernel_launches()
    sampler.start()
    ms, agg = timed(batched_step, args.steps)
    clocks = sampler.stop()
    launches = A.kernel_launches() - launches0
    if args.profile:
        if rank == 0:
            print(json.dumps({"profile_run": True, "ms_per_step": ms, "queries": Q, "launches": launches // args.steps}))
        return
    # the plain form, for the batched / plain ratio
    for _ in range(max(1, args.warmup // 2)):
        plain_step()
    plain_ms, plain_agg = timed(plain_step, args.steps)
    learned = None
    if est is not None:
        # the planner (exhaustive prefix search or greedy) for learned estimates, on the tuned kernel knobs
        learned_tune, learned_table = A.autotune(
            dg, packed, min_blocks=(tune_best["enum_min_blocks"],), lane_leaf=(tune_best["lane_leaf_max"],),
            run=lambda d, b: A.run_batch_ex(d, b, estimator=est, learned_max_subset=args.learned_max))
        for _ in range(max(1, args.warmup // 2)):
            learned_step()
        learned_ms, learned_agg = timed(learned_step, args.steps)
        learned = {"queries_per_s": world * Q / (learned_ms / 1e3), "ms_per_step": learned_ms,
                   "enum_kernel_ms_per_step": learned_agg["kernel_ms"] / args.steps,
                   "cs_build_ms_per_step": learned_agg["cs_ms"] / args.steps,
                   "intersections_per_step": learned_agg["inter"] // args.steps,
                   "over_plain": plain_ms / learned_ms, "over_cost_model_batched": ms / learned_ms,
                   "estimator": os.path.relpath(est_path, ROOT) if est_path.startswith(ROOT) else est_path,
                   "learned_max_subset": args.learned_max or 6,
                   "planner": "exhaustive prefix search" if learned_tune["planner"] == A.PLANNER_DP else "greedy",
                   "planner_table": learned_table,
                   "what": "asdm_run_batch_ex with the learned estimator: candidate spaces, learned greedy plans "
                           "(one forward pass per planner step for the whole group), one persistent launch; "
                           "planning is inside the timed region"}
        dg.set_tuning(tune_best["enum_min_blocks"], tune_best["lane_leaf_max"], tune_best["planner"],
                      tune_best["root_block_min"])
    # end to end through the one-call C ABI (asdm_run_batch) from host buffers
    e2e_times = []
    h2d = packed.nbytes()
    d2h = Q * (8 + 4)
    for _ in range(args.steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        A.run_batch_packed(dg, packed)
        e2e_times.append(time.perf_counter() - t0)
        if packed.counts.tolist() != counts or packed.status.any():
            raise SystemExit("batch counts differ from the screened counts")
    e2e_s = max_over_ranks(statistics.mean(e2e_times), world, dev)
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    peak, peak_kind = measured_peaks()
    steps = args.steps
    enum_ms, cs_ms = agg["kernel_ms"] / steps, agg["cs_ms"] / steps
    # the largest single kernel of the step is the enumeration launch; the
    # candidate-space build (a dozen smaller launches) gets its own line
    dom, bytes_, kms = "enum_batch_kernel (K4-K8 warp DFS, batched)", agg["list_bytes"] / steps, enum_ms
    achieved = bytes_ / (kms * 1e-3) / 1e9 if kms > 0 else 0.0
    cs_bytes = agg["cs_bytes"] / steps
    cs_achieved = cs_bytes / (cs_ms * 1e-3) / 1e9 if cs_ms > 0 else 0.0
    traffic = traffic_cs = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as fh:
            t = json.load(fh).get(args.workload) or {}
        traffic, traffic_cs = t.get("enum_batch_kernel"), t.get("k1_k3")
    line = {
        "metric": "exact-count queries/sec",
        "value": world * Q / (ms / 1e3),
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
                       form="batched: asdm_run_batch (one launch per CFL phase for the group, one persistent "
                            "enumeration kernel over all (query, root task) pairs); planner: candidate-size cost model, "
                            + ("exhaustive prefix search" if tune_best.get("planner", 0) == A.PLANNER_DP else "greedy"),
                       matches_per_step=agg["matches"] // steps,
                       matches_per_s=world * (agg["matches"] // steps) / (ms / 1e3),
                       intersections_per_step=agg["inter"] // steps,
                       enum_kernel_ms_per_step=enum_ms, cs_build_ms_per_step=cs_ms,
                       plain_form={"queries_per_s": world * Q / (plain_ms / 1e3), "ms_per_step": plain_ms,
                                   "enum_kernel_ms_per_step": plain_agg["kernel_ms"] / steps,
                                   "cs_build_ms_per_step": plain_agg["cs_ms"] / steps,
                                   "what": "one query per launch sequence (asdm_candidate_space, asdm_plan_create, "
                                           "asdm_run_plan)"},
                       batched_over_plain=plain_ms / ms,
                       cs_build_roofline={"kernels": "K1-K3 (k1_filter, k2_pull, compaction, k3_bound/flat/pack)",
                                          "bound": "hbm", "achieved": cs_achieved, "peak": peak, "unit": "GB/s",
                                          "frac": cs_achieved / peak, "algorithmic_bytes_per_step": cs_bytes,
                                          "device_ms_per_step": cs_ms, "traffic": traffic_cs},
                       batched_learned=learned,
                       autotune={"chosen": tune_best, "table": tune_table}),
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "algorithmic_bytes_per_step": bytes_, "device_ms_per_step": kms, "traffic": traffic},
        "e2e": {"value": world * Q / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "via": "asdm_run_batch (C ABI) from host arrays, wall clock"},
        "gpu_launches": launches // steps,
        "clocks": clocks,
    }
    # config 4: batched local subgraph counting (LOCAL_COUNT), secondary measurement
    if world == 1 and not args.no_c4 and os.path.exists(W.C4_SCREEN_FILE):
        line["config"]["local_counting_c4"] = measure_c4(A, W, torch, dev, args.steps)
    if world == 1:
        tmp = tempfile.mkdtemp(prefix="asdm_cpu_")
        dpath = os.path.join(tmp, "data.graph")
        g.write(dpath)
        order = sorted(range(Q), key=lambda i: counts[i])  # smallest counts first keeps the sample bounded
        sample = order[len(order) // 2: len(order) // 2 + args.cpu_sample]
        qpaths = []
        for i in sample:
            p = os.path.join(tmp, "q%d.graph" % i)
            qs[i].write(p)
            qpaths.append(p)
        line["cpu_baseline"] = cpu_baseline(dpath, qpaths, [counts[i] for i in sample])
    print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
