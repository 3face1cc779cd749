"""CPU results for the config-2 batch (tests/golden/c2_batch.json).

    python tests/golden/make_c2_golden.py reference [--cap S] [--jobs J] [--sizes LO-HI]
    python tests/golden/make_c2_golden.py oracle [--jobs J]
    python tests/golden/make_c2_golden.py bounds [--jobs J]

The config-2 batch is the first 1,000 random-walk queries (seeds 50,000 + i,
sizes uniform in 4..32) on the config-1 graph.  Inputs are written by the
host-only generator (asdmatch_b200/bin/asdm_gen.out) into --workdir.

* reference: the reference's own ALL_LEVEL build (oracle/_ref/ref_count,
  compiled from the reference sources by oracle/ref.mk) on each query of the
  size range, one forked process per query after one graph load, killed at
  the cap; records the reference's count and 'Execution Time' where it
  finished ("count"), or that it did not ("reference": "timeout").
* oracle: the CPU oracle (oracle/_build/asdm_oracle) on every tree query:
  its inclusion-exclusion count ("oracle_tree": a count, "overflow" for a
  count of 2^64 or more, or "skip" where a quotient has a cycle); and on the
  parity set (two queries of every size 7..32, "parity") its restatement of
  the device's overflow lower bound ("oracle_bound").
* bounds: the oracle's lower bounds of the parity set alone.

Runs merge into the same file (a finished reference count is never replaced
by a later timeout).  --reuse DIR merges the outputs a previous run of the
same step left in DIR instead of running it again.
"""
import argparse
import importlib.util
import json
import os
import subprocess
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "c2_batch.json")
REF = os.path.join(ROOT, "oracle", "_ref", "ref_count")
ORACLE = os.path.join(ROOT, "oracle", "_build", "asdm_oracle")
GEN = os.path.join(ROOT, "asdmatch_b200", "bin", "asdm_gen.out")


def specs():
    spec = importlib.util.spec_from_file_location("asdm_specs", os.path.join(ROOT, "asdmatch_b200", "specs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def parity_set(S):
    """Two queries of every size from 7 to 32: the first two in batch order."""
    out = []
    for size in range(7, 33):
        out += [i for i in range(S.C2_QUERIES) if S.c2_seed_size(i)[1] == size][:2]
    return out


def write_inputs(S, workdir, idx):
    os.makedirs(workdir, exist_ok=True)
    dpath = os.path.join(workdir, "data.graph")
    if not os.path.exists(dpath):
        subprocess.run([GEN, "graph"] + S.generator_args(S.C1) + [dpath], check=True)
    missing = [i for i in idx if not os.path.exists(os.path.join(workdir, "q%d.graph" % i))]
    if missing:
        gl = os.path.join(workdir, "gen.txt")
        with open(gl, "w") as fh:
            for i in missing:
                seed, size = S.c2_seed_size(i)
                fh.write("%d %d 0 q%d.graph\n" % (size, seed, i))
        subprocess.run([GEN, "queries"] + S.generator_args(S.C1) + [gl, workdir], check=True)
    return dpath


def is_tree(path):
    with open(path) as fh:
        _, n, m = fh.readline().split()[:3]
    return int(m) == int(n) - 1


def load():
    if os.path.exists(OUT):
        with open(OUT) as fh:
            return json.load(fh)
    return {"queries": []}


def save(data, S):
    data["queries"].sort(key=lambda r: r["index"])
    data["parity"] = parity_set(S)
    data["how"] = {
        "count": "reference ALL_LEVEL build (oracle/_ref/ref_count), one forked process per query after one graph "
                 "load, killed at cap_s; its 'Number of matches' where it finished",
        "oracle_tree": "asdm_oracle -t: inclusion-exclusion over same-label blocks, 128-bit integers",
        "oracle_bound": "asdm_oracle -b: the device's overflow lower bound restated from its definition"}
    with open(OUT, "w") as fh:
        json.dump(data, fh, indent=0)


def record(data, S, i):
    have = {r["index"]: r for r in data["queries"]}
    if i not in have:
        seed, size = S.c2_seed_size(i)
        rec = {"index": i, "seed": seed, "size": size, "count": None}
        data["queries"].append(rec)
        return rec
    return have[i]


def run_reference(args, S, data):
    lo, hi = (int(x) for x in args.sizes.split("-"))
    idx = [i for i in range(S.C2_QUERIES) if lo <= S.c2_seed_size(i)[1] <= hi]
    dpath = write_inputs(S, args.workdir, idx)
    if args.reuse:
        outdir = args.reuse
        paths = open(os.path.join(outdir, "list.txt")).read().split()
        lines = open(os.path.join(outdir, "status.txt")).read().splitlines()
    else:
        outdir = os.path.join(args.workdir, "ref_%d_%d" % (lo, hi))
        os.makedirs(outdir, exist_ok=True)
        paths = [os.path.join(args.workdir, "q%d.graph" % i) for i in idx]
        with open(os.path.join(outdir, "list.txt"), "w") as fh:
            fh.write("\n".join(paths) + "\n")
        t0 = time.time()
        r = subprocess.run([REF, "-d", dpath, "-Q", os.path.join(outdir, "list.txt"), "-O", outdir,
                            "-T", str(args.cap), "-J", str(args.jobs)], capture_output=True, text=True, check=True)
        lines = r.stdout.splitlines()
        with open(os.path.join(outdir, "status.txt"), "w") as fh:
            fh.write(r.stdout)
        print("reference runs: %.0f s" % (time.time() - t0))
    for line in lines:
        parts = line.split()
        if len(parts) < 4 or parts[0] != "Q":
            continue
        k = int(parts[1])
        i = int(os.path.basename(paths[k])[1:].split(".")[0])
        rec = record(data, S, i)
        if rec.get("count") is not None:
            continue
        rec.update(reference=parts[2], cap_s=args.cap, wall_s=round(float(parts[-1]), 3))
        if parts[2] == "ok":
            for l in open(os.path.join(outdir, "q%d.out" % k)):
                if l.startswith("Number of matches:"):
                    rec["count"] = int(l.split(":")[1])
                elif l.startswith("Execution Time:"):
                    rec["execution_s"] = float(l.split(":")[1])


def run_oracle_lists(dpath, lists, flag, jobs):
    """asdm_oracle <flag> over the list files, `jobs` processes at a time."""
    procs = [subprocess.Popen([ORACLE, "-d", dpath, flag, lst], stdout=subprocess.PIPE, text=True) for lst in lists]
    return [p.communicate()[0] for p in procs]


def write_list(path, workdir, idx):
    with open(path, "w") as fh:
        fh.write("\n".join(os.path.join(workdir, "q%d.graph" % i) for i in idx) + "\n")
    return path


def run_bounds(args, S, data):
    """asdm_oracle -b on the parity set, split over --jobs processes."""
    par = parity_set(S)
    dpath = write_inputs(S, args.workdir, par)
    jobs = max(1, min(args.jobs, len(par)))
    parts = [par[k::jobs] for k in range(jobs)]
    lists = [write_list(os.path.join(args.workdir, "parity_list_%d.txt" % k), args.workdir, part)
             for k, part in enumerate(parts)]
    for part, text in zip(parts, run_oracle_lists(dpath, lists, "-b", jobs)):
        for line in text.splitlines():
            f = line.split()
            if len(f) == 3 and f[0] == "B":
                record(data, S, part[int(f[1])])["oracle_bound"] = f[2]


def run_oracle(args, S, data):
    idx = list(range(S.C2_QUERIES))
    dpath = write_inputs(S, args.workdir, idx)
    trees = [i for i in idx if is_tree(os.path.join(args.workdir, "q%d.graph" % i))]
    jobs = max(1, args.jobs)
    if args.reuse:
        outs = [(json.load(open(os.path.join(args.reuse, "tree_list_%d.json" % k))),
                 open(os.path.join(args.reuse, "tree_out_%d.txt" % k)).read()) for k in range(jobs)]
    else:
        parts = [trees[k::jobs] for k in range(jobs)]
        lists = [write_list(os.path.join(args.workdir, "tree_list_%d.txt" % k), args.workdir, part)
                 for k, part in enumerate(parts)]
        outs = list(zip(parts, run_oracle_lists(dpath, lists, "-t", jobs)))
    for part, text in outs:
        for line in text.splitlines():
            f = line.split()
            if len(f) < 3 or f[0] != "T":
                continue
            rec = record(data, S, part[int(f[1])])
            rec["oracle_tree"] = int(f[3]) if f[2] == "ok" else ("overflow" if f[2] == "overflow" else
                                                                  (0 if f[2] == "empty" else "skip"))
    run_bounds(args, S, data)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("step", choices=["reference", "oracle", "bounds"])
    ap.add_argument("--cap", type=float, default=60.0)
    ap.add_argument("--jobs", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    ap.add_argument("--sizes", default="4-32")
    ap.add_argument("--workdir", default=os.path.join(ROOT, "_work", "c2ref"))
    ap.add_argument("--reuse", default="")
    args = ap.parse_args()
    S = specs()
    data = load()
    if args.step == "reference":
        run_reference(args, S, data)
    elif args.step == "bounds":
        run_bounds(args, S, data)
    else:
        run_oracle(args, S, data)
    save(data, S)
    fin = sum(1 for r in data["queries"] if r.get("count") is not None)
    tr = sum(1 for r in data["queries"] if isinstance(r.get("oracle_tree"), int))
    print("c2 golden: %d queries, %d reference counts, %d oracle tree counts" % (len(data["queries"]), fin, tr))


if __name__ == "__main__":
    main()
