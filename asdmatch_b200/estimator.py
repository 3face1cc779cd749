"""Training and evaluation of the learned cardinality estimator.

The reference plans with subset cardinalities it estimates by sampling partial
matches inside the candidate space (cardEstimateLabeled,
plan/estimator.cpp:173-291, stored in subsetToCard, plan/estimator.cpp:7).
Here the engine counts those partial matches exactly (``prefix_counts``: one
batched launch per query), the counts become training targets
log(1 + count) for the device-side message-passing network
(``asdmatch_b200.Estimator``), and the trained network feeds the planner
(``run_batch_ex(..., estimator=...)`` / ``plans_learned``).  Features are
computed by the library (``subset_features``), identically for training and
planning.

Workload (the reference's training-set shape): random-walk queries of 4..24
vertices on the config-1 graph, 3..6-vertex connected sub-queries sampled from
each; a disjoint set of queries is held out for the q-error.
"""
from __future__ import annotations

import json
import os
import time
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

import asdmatch_b200 as A

TRAIN_QUERY_SEED = 200_000
HELDOUT_QUERY_SEED = 300_000
COUNT_LIMIT = 10 ** 9
DEFAULT_PARAMS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "estimator_c1.npy")
DEFAULT_REPORT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "estimator_c1.json")


def query_adjacency(q: A.HostGraph) -> List[List[int]]:
    off = q.offsets.astype(np.int64)
    return [q.nbrs[off[u]:off[u + 1]].tolist() for u in range(q.n)]


def sample_subsets(q: A.HostGraph, rng: np.random.Generator, count: int, kmin: int = 3, kmax: int = 6) -> List[int]:
    """Up to `count` distinct connected vertex subsets (bitmasks) of kmin..kmax
    vertices, grown from a random vertex by random frontier steps."""
    if q.n < kmin:
        return []
    adj = query_adjacency(q)
    out, tries = set(), 0
    while len(out) < count and tries < 20 * count:
        tries += 1
        k = int(rng.integers(kmin, min(kmax, q.n) + 1))
        start = int(rng.integers(q.n))
        chosen, mask = [start], 1 << start
        frontier = set(adj[start])
        while len(chosen) < k and frontier:
            w = int(rng.choice(sorted(frontier)))
            chosen.append(w)
            mask |= 1 << w
            frontier |= set(adj[w])
            frontier -= set(chosen)
        if len(chosen) == k:
            out.add(mask)
    return sorted(out)


def connected_subsets(q: A.HostGraph, kmax: int) -> List[int]:
    """Every connected vertex subset of 1..kmax vertices (the ESU enumeration)."""
    adj = query_adjacency(q)
    out = []

    def extend(sub, ext, v, mask):
        out.append(mask)
        if len(sub) == kmax:
            return
        ext = list(ext)
        while ext:
            w = ext.pop()
            new_ext = list(ext)
            nb = set(sub)
            for s in sub:
                nb.update(adj[s])
            for x in adj[w]:
                if x > v and x not in nb and x not in new_ext:
                    new_ext.append(x)
            extend(sub + [w], new_ext, v, mask | (1 << w))

    for v in range(q.n):
        extend([v], [x for x in adj[v] if x > v], v, 1 << v)
    return out


def connected_order(adj: List[List[int]], mask: int) -> List[int]:
    """A breadth-first order of the subset `mask` from its lowest vertex."""
    start = (mask & -mask).bit_length() - 1
    order, seen = [start], {start}
    i = 0
    while i < len(order):
        for w in adj[order[i]]:
            if mask >> w & 1 and w not in seen:
                seen.add(w)
                order.append(w)
        i += 1
    return order


@dataclass
class Dataset:
    """Samples (sub-queries) packed node-major."""
    x: List[np.ndarray] = field(default_factory=list)        # per sample: nodes x EST_FEATURES
    nbr: List[List[np.ndarray]] = field(default_factory=list)  # per sample: per node local neighbours
    y: List[float] = field(default_factory=list)             # log(1 + count)
    censored: List[bool] = field(default_factory=list)       # count reached the limit (y is a floor)
    sampled: List[float] = field(default_factory=list)       # log(1 + sampling estimate), or nan
    sampled_targets: bool = False                            # censored samples take the sampling estimate as y
    size: List[int] = field(default_factory=list)
    query: List[int] = field(default_factory=list)

    def __len__(self):
        return len(self.y)

    def add_query(self, cs: A.CandidateSpace, masks: Sequence[int], counts, status, qid: int,
                  count_limit: int = COUNT_LIMIT, sampled=None):
        keep = [i for i in range(len(masks)) if status[i] in (A.OK, A.ERR_LIMIT)]
        if not keep:
            return
        sel = [masks[i] for i in keep]
        x, off, adj, gid = A.subset_features(cs, sel)
        starts = np.searchsorted(gid, np.arange(len(sel)))
        ends = np.append(starts[1:], len(gid))
        for j, i in enumerate(keep):
            s, e = int(starts[j]), int(ends[j])
            self.x.append(x[s:e].copy())
            self.nbr.append([adj[off[v]:off[v + 1]].astype(np.int64) - s for v in range(s, e)])
            lim = status[i] == A.ERR_LIMIT
            y = float(np.log1p(float(count_limit if lim else counts[i])))
            if lim and sampled is not None and self.sampled_targets:
                # past the exact-count limit the sampling estimate is the target (never below the floor)
                y = max(y, float(np.log1p(sampled[i])))
            self.y.append(y)
            self.censored.append(bool(lim))
            self.sampled.append(float(np.log1p(sampled[i])) if sampled is not None else float("nan"))
            self.size.append(e - s)
            self.query.append(qid)

    def batch(self, idx: Sequence[int]):
        """(x, adj_off, adj, node_graph, y) for the samples idx."""
        xs, offs, adjs, gids = [], [0], [], []
        base = 0
        for g, i in enumerate(idx):
            xs.append(self.x[i])
            for nb in self.nbr[i]:
                adjs.append(nb + base)
                offs.append(offs[-1] + len(nb))
            gids.append(np.full(len(self.x[i]), g, np.uint32))
            base += len(self.x[i])
        adj = np.concatenate(adjs).astype(np.uint32) if adjs else np.zeros(0, np.uint32)
        return (np.concatenate(xs), np.asarray(offs, np.uint32), adj, np.concatenate(gids),
                np.asarray([self.y[i] for i in idx], np.float32))

    def independence(self, i: int) -> float:
        """log of the planner-style independence estimate: 16 x sum of feature 39."""
        return float(16.0 * self.x[i][:, 39].sum())


def collect(dg: A.DeviceGraph, queries: Sequence[A.HostGraph], rng: np.random.Generator, per_query: int = 24,
            kmin: int = 3, kmax: int = 6, time_limit_s: float = 5.0, chunk: int = 64, qid0: int = 0,
            log=None, count_limit: int = COUNT_LIMIT, walks: int = 0, sampled_targets: bool = False) -> Dataset:
    """Exact partial-match counts of sampled sub-queries inside each query's
    candidate space (counts at or above count_limit are kept as censored);
    with walks > 0 also the sampling estimator's estimates of the same
    sub-queries (asdm_sample_subsets), which with sampled_targets become the
    targets of the censored samples."""
    ds = Dataset(sampled_targets=sampled_targets)
    for at in range(0, len(queries), chunk):
        part = list(queries[at:at + chunk])
        css = A.candidate_spaces(dg, part)
        for j, (q, cs) in enumerate(zip(part, css)):
            if cs is None or not cs.nonempty:
                continue
            masks = sample_subsets(q, rng, per_query, kmin, kmax)
            if not masks:
                continue
            adj = query_adjacency(q)
            orders = [connected_order(adj, m) for m in masks]
            counts, status = cs.prefix_counts(orders, time_limit_s=time_limit_s, count_limit=count_limit)
            sampled = cs.sample_cardinalities(masks, walks, seed=qid0 + at + j) if walks else None
            ds.add_query(cs, masks, counts, status, qid0 + at + j, count_limit, sampled)
        del css
        if log:
            log("collected %d queries, %d samples" % (min(at + chunk, len(queries)), len(ds)))
    return ds


def train(est: A.Estimator, ds: Dataset, epochs: int = 40, batch: int = 256, lr: float = 1e-3, seed: int = 0,
          log=None) -> List[float]:
    rng = np.random.default_rng(seed)
    losses = []
    n = len(ds)
    for ep in range(epochs):
        perm = rng.permutation(n)
        tot, nb = 0.0, 0
        step_lr = lr * (0.5 * (1 + np.cos(np.pi * ep / epochs)) * 0.9 + 0.1)  # cosine to lr/10
        for at in range(0, n, batch):
            idx = perm[at:at + batch]
            x, off, adj, gid, y = ds.batch(idx)
            tot += est.train_step(x, off, adj, gid, y, lr=float(step_lr))
            nb += 1
        losses.append(tot / max(nb, 1))
        if log and (ep % 5 == 0 or ep == epochs - 1):
            log("epoch %d loss %.4f" % (ep, losses[-1]))
    return losses


def predict(est: A.Estimator, ds: Dataset, batch: int = 4096) -> np.ndarray:
    out = []
    for at in range(0, len(ds), batch):
        idx = list(range(at, min(len(ds), at + batch)))
        x, off, adj, gid, _ = ds.batch(idx)
        out.append(est.predict(x, off, adj, gid, len(idx)))
    return np.concatenate(out) if out else np.zeros(0, np.float32)


def q_errors(pred_log: np.ndarray, true_log: np.ndarray) -> np.ndarray:
    """max(est/true, true/est) with both cardinalities floored at 1."""
    p = np.maximum(np.expm1(np.clip(pred_log, 0, 60)), 1.0)
    t = np.maximum(np.expm1(true_log), 1.0)
    return np.maximum(p / t, t / p)


def evaluate(est: A.Estimator, ds: Dataset) -> dict:
    """q-errors of the learned estimates (and of the planner's independence
    estimate, and of the sampling estimator where the samples carry its
    estimates) against the exact counts; for censored samples (counts past the
    limit) the sampling estimator is the judge of the learned estimates."""
    pred = predict(est, ds)
    y = np.asarray(ds.y)
    exact = ~np.asarray(ds.censored, bool)
    q = q_errors(pred[exact], y[exact])
    ind = np.asarray([ds.independence(i) for i in range(len(ds))])
    qi = q_errors(np.log1p(np.exp(np.clip(ind[exact], -50, 60))), y[exact])

    def pct(a):
        return {"p50": float(np.percentile(a, 50)), "p90": float(np.percentile(a, 90)),
                "p99": float(np.percentile(a, 99)), "mean": float(np.mean(a))} if len(a) else {}

    out = {"samples": int(exact.sum()), "censored": int((~exact).sum()), "learned": pct(q),
           "independence": pct(qi)}
    smp = np.asarray(ds.sampled, np.float64)
    if len(smp) and np.isfinite(smp).any():
        have = np.isfinite(smp)
        out["sampling"] = pct(q_errors(smp[exact & have], y[exact & have]))
        cen = ~exact & have
        out["censored_learned_vs_sampling"] = pct(q_errors(pred[cen], smp[cen]))
    return out


def queries_c3(g: A.HostGraph, count: int, seed0: int) -> List[A.HostGraph]:
    """Random-walk queries of 4..24 vertices (uniform), seeds seed0 + i."""
    out = []
    for i in range(count):
        seed = seed0 + i
        size = 4 + (seed * 2654435761 % 2 ** 32) % 21
        out.append(g.random_walk_query(size, seed, 0))
    return out


def load(path: str = DEFAULT_PARAMS, seed: int = 0) -> A.Estimator:
    est = A.Estimator(A.EST_FEATURES, seed)
    est.set_params(np.load(path))
    return est


def main(argv=None):
    import argparse
    import asdmatch_b200.workloads as W
    ap = argparse.ArgumentParser(description="train the learned estimator on the config-1 graph")
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--heldout", type=int, default=200)
    ap.add_argument("--per-query", type=int, default=24)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--out", default=DEFAULT_PARAMS)
    ap.add_argument("--report", default=DEFAULT_REPORT)
    ap.add_argument("--eval-only", default="", help="evaluate these trained parameters on the held-out queries")
    ap.add_argument("--count-limit", type=int, default=COUNT_LIMIT, help="exact counts past this are censored")
    ap.add_argument("--walks", type=int, default=4096, help="sampling-estimator walks per held-out sub-query")
    ap.add_argument("--train-walks", type=int, default=1024,
                    help="sampling-estimator walks per training sub-query (targets of the censored ones; 0: floors)")
    a = ap.parse_args(argv)
    t0 = time.time()
    g = W.graph(W.C1)
    dg = A.DeviceGraph(g)
    rng = np.random.default_rng(7)
    if a.eval_only:
        # the held-out set alone: learned, sampling and independence estimates against exact counts
        est = load(a.eval_only)
        hq = queries_c3(g, a.heldout, HELDOUT_QUERY_SEED)
        hs = collect(dg, hq, rng, a.per_query, qid0=10 ** 6, log=print, count_limit=a.count_limit,
                     time_limit_s=20.0, walks=a.walks)
        rep = {"graph": W.C1, "params": os.path.basename(a.eval_only), "heldout_queries": a.heldout,
               "per_query": a.per_query, "heldout_seed": HELDOUT_QUERY_SEED, "count_limit": a.count_limit,
               "walks": a.walks, "collect_s": time.time() - t0, "heldout_eval": evaluate(est, hs)}
        with open(a.report, "w") as fh:
            json.dump(rep, fh, indent=1)
        print(json.dumps(rep["heldout_eval"]))
        return
    tq = queries_c3(g, a.train, TRAIN_QUERY_SEED)
    hq = queries_c3(g, a.heldout, HELDOUT_QUERY_SEED)
    t1 = time.time()
    # training targets: exact counts up to COUNT_LIMIT, sampling estimates past it; held out:
    # exact counts up to --count-limit, with the sampling estimator's estimates beside them
    ds = collect(dg, tq, rng, a.per_query, log=print, walks=a.train_walks, sampled_targets=a.train_walks > 0)
    hs = collect(dg, hq, rng, a.per_query, qid0=10 ** 6, log=print, count_limit=a.count_limit,
                 time_limit_s=20.0, walks=a.walks)
    t2 = time.time()
    est = A.Estimator(A.EST_FEATURES, 1)
    losses = train(est, ds, epochs=a.epochs, log=print)
    t3 = time.time()
    rep = {"graph": W.C1, "train_queries": a.train, "heldout_queries": a.heldout, "per_query": a.per_query,
           "train_seed": TRAIN_QUERY_SEED, "heldout_seed": HELDOUT_QUERY_SEED, "count_limit": COUNT_LIMIT,
           "heldout_count_limit": a.count_limit, "train_walks": a.train_walks, "heldout_walks": a.walks,
           "train_targets": "exact counts up to count_limit, sampling estimates past it" if a.train_walks else
                            "exact counts up to count_limit, count_limit past it",
           "train_samples": len(ds), "epochs": a.epochs, "final_loss": losses[-1],
           "collect_s": t2 - t1, "train_s": t3 - t2, "setup_s": t1 - t0,
           "train_eval": evaluate(est, ds), "heldout_eval": evaluate(est, hs)}
    np.save(a.out, est.params())
    with open(a.report, "w") as fh:
        json.dump(rep, fh, indent=1)
    print(json.dumps(rep["heldout_eval"]))


if __name__ == "__main__":
    main()
