"""Reference counts of the config-2 batch (tests/golden/c2_batch.json).

    python tests/golden/make_c2_golden.py [--cap S] [--jobs J] [--sizes LO-HI] [--workdir DIR]

The config-2 batch is the first 1,000 random-walk queries (seeds 50,000 +
i, sizes uniform in 4..32) on the config-1 graph.  This script writes the
graph and the queries with the host-only generator (asdmatch_b200/bin/
asdm_gen.out), runs the reference's own ALL_LEVEL build (oracle/_ref/
ref_count, compiled from the reference sources by oracle/ref.mk) on each query
in its own process with a time cap, and records per query either the
reference's exact count with its 'Execution Time', or that it did not finish
within the cap.  Runs over several size ranges merge into the same file (a
finished query is never overwritten by a later timeout).
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
GEN = os.path.join(ROOT, "asdmatch_b200", "bin", "asdm_gen.out")


def specs():
    spec = importlib.util.spec_from_file_location("asdm_specs", os.path.join(ROOT, "asdmatch_b200", "specs.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cap", type=float, default=60.0)
    ap.add_argument("--jobs", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    ap.add_argument("--sizes", default="4-32")
    ap.add_argument("--workdir", default=os.path.join(ROOT, "_work", "c2ref"))
    ap.add_argument("--outputs", default="", help="reuse a finished harness run: its list file and output dir")
    args = ap.parse_args()
    S = specs()
    lo, hi = (int(x) for x in args.sizes.split("-"))
    idx = [i for i in range(S.C2_QUERIES) if lo <= S.c2_seed_size(i)[1] <= hi]
    os.makedirs(args.workdir, exist_ok=True)
    dpath = os.path.join(args.workdir, "data.graph")
    if not os.path.exists(dpath):
        subprocess.run([GEN, "graph"] + S.generator_args(S.C1) + [dpath], check=True)
    gl = os.path.join(args.workdir, "gen.txt")
    with open(gl, "w") as fh:
        for i in idx:
            seed, size = S.c2_seed_size(i)
            fh.write("%d %d 0 q%d.graph\n" % (size, seed, i))
    subprocess.run([GEN, "queries"] + S.generator_args(S.C1) + [gl, args.workdir], check=True)
    if args.outputs:
        lst, outdir = args.outputs.split(",")
        status_lines = open(os.path.join(outdir, "status.txt")).read().splitlines()
    else:
        outdir = os.path.join(args.workdir, "out_%d_%d" % (lo, hi))
        os.makedirs(outdir, exist_ok=True)
        lst = os.path.join(outdir, "list.txt")
        with open(lst, "w") as fh:
            fh.write("\n".join(os.path.join(args.workdir, "q%d.graph" % i) for i in idx) + "\n")
        t0 = time.time()
        r = subprocess.run([REF, "-d", dpath, "-Q", lst, "-O", outdir, "-T", str(args.cap), "-J", str(args.jobs)],
                           capture_output=True, text=True, check=True)
        status_lines = r.stdout.splitlines()
        print("reference runs: %.0f s" % (time.time() - t0))
    paths = open(lst).read().split()
    data = {"queries": []}
    if os.path.exists(OUT):
        with open(OUT) as fh:
            data = json.load(fh)
    have = {r["index"]: r for r in data["queries"]}
    for line in status_lines:
        parts = line.split()
        if len(parts) < 4 or parts[0] != "Q":
            continue
        k = int(parts[1])
        i = int(os.path.basename(paths[k])[1:].split(".")[0])
        seed, size = S.c2_seed_size(i)
        rec = {"index": i, "seed": seed, "size": size, "count": None, "reference": parts[2],
               "cap_s": args.cap, "wall_s": round(float(parts[-1]), 3)}
        if parts[2] == "ok":
            for l in open(os.path.join(outdir, "q%d.out" % k)):
                if l.startswith("Number of matches:"):
                    rec["count"] = int(l.split(":")[1])
                elif l.startswith("Execution Time:"):
                    rec["execution_s"] = float(l.split(":")[1])
        old = have.get(i)
        if old is None or old.get("count") is None:
            have[i] = rec
    data["queries"] = [have[i] for i in sorted(have)]
    data["how"] = ("reference ALL_LEVEL build (oracle/_ref/ref_count) per query, one forked process each after one "
                   "graph load, killed at cap_s; count = its 'Number of matches' where it finished")
    with open(OUT, "w") as fh:
        json.dump(data, fh, indent=0)
    fin = sum(1 for r in data["queries"] if r["count"] is not None)
    print("c2 golden: %d queries recorded, %d with reference counts" % (len(data["queries"]), fin))


if __name__ == "__main__":
    main()
