"""Reference results for the config-4 graph (tests/golden/c4_batch.json).

    python tests/golden/make_c4_golden.py [--cap S] [--jobs J] [--parity-only]

Config 4 is local subgraph counting: the Chung-Lu graph N=1.0M, M=10M,
exponent 2.3, 32 labels Zipf(1.0).  Two query sets:
* "queries": the 50 random-walk queries of 10 vertices of the configuration
  (seeds 90,000 + i);
* "parity": 40 random-walk queries of 4..8 vertices (seeds 95,000 + i), small
  enough for the reference to finish, so that its CSV can be compared at the
  graph's full size (tests/test_gpu_c4_parity.py);
* "embed": 16 dense random-walk queries of 5..8 vertices (the first seeds from
  96,000 whose walk gives a dense query), whose sorted embedding sets the
  reference's COLLECT_RESULT build dumps (oracle/_ref/ref_embed).
This script writes them with the host-only generator
(asdmatch_b200/bin/asdm_gen.out) and runs the reference's ALL_LEVEL +
LOCAL_COUNT build (oracle/_ref/ref_local) on each query in its own forked
process after one graph load, killed at the cap.  Where the reference
finished it records the count and the SHA-256 of the |Vg| x |Vq| CSV it wrote
(main.cpp:135-146); otherwise that it did not finish.  --parity-only keeps the
recorded "queries" and recomputes "parity" and "embed";
--embed-only recomputes "embed" alone.
"""
import argparse
import hashlib
import importlib.util
import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "c4_batch.json")
REF = os.path.join(ROOT, "oracle", "_ref", "ref_local")
GEN = os.path.join(ROOT, "asdmatch_b200", "bin", "asdm_gen.out")


def run_reference(S, specs, workdir, name, dpath, cap, jobs):
    qdir = os.path.join(workdir, name)
    os.makedirs(qdir, exist_ok=True)
    gl = os.path.join(qdir, "gen.txt")
    with open(gl, "w") as fh:
        for k, (size, seed, density) in enumerate(specs):
            fh.write("%d %d %d q%d.graph\n" % (size, seed, density, k))
    subprocess.run([GEN, "queries"] + S.generator_args(S.C4) + [gl, qdir], check=True)
    outdir = os.path.join(qdir, "out")
    os.makedirs(outdir, exist_ok=True)
    lst = os.path.join(outdir, "list.txt")
    with open(lst, "w") as fh:
        fh.write("\n".join(os.path.join(qdir, "q%d.graph" % k) for k in range(len(specs))) + "\n")
    r = subprocess.run([REF, "-d", dpath, "-Q", lst, "-O", outdir, "-T", str(cap), "-J", str(jobs),
                        "-c", "csv"], capture_output=True, text=True, check=True)
    recs = []
    for line in r.stdout.splitlines():
        f = line.split()
        if len(f) < 4 or f[0] != "Q":
            continue
        k = int(f[1])
        size, seed, density = specs[k]
        rec = {"index": k, "seed": seed, "size": size, "reference": f[2], "cap_s": cap,
               "wall_s": round(float(f[-1]), 3), "count": None}
        if f[2] == "ok":
            for l in open(os.path.join(outdir, "q%d.out" % k)):
                if l.startswith("Number of matches:"):
                    rec["count"] = int(l.split(":")[1])
            h = hashlib.sha256()
            with open(os.path.join(outdir, "q%d.csv" % k), "rb") as fh:
                for chunk in iter(lambda: fh.read(1 << 20), b""):
                    h.update(chunk)
            rec["csv_sha256"] = h.hexdigest()
        recs.append(rec)
    recs.sort(key=lambda x: x["index"])
    return recs


def embed_queries(workdir, want=16):
    """Dense random-walk queries of 5..8 vertices on the config-4 graph (seeds
    from C4_EMBED_SEED upwards; a seed whose walk gives no dense query is
    skipped), written to <workdir>/embed/q<k>.graph; returns their
    (size, seed, density) specs."""
    import sys
    sys.path.insert(0, ROOT)
    import asdmatch_b200 as A
    from asdmatch_b200 import specs as SP
    from asdmatch_b200 import workloads as W
    g = W.graph(W.C4)
    qdir = os.path.join(workdir, "embed")
    os.makedirs(qdir, exist_ok=True)
    specs, seed = [], SP.C4_EMBED_SEED
    while len(specs) < want:
        size = 5 + len(specs) % 4
        try:
            q = g.random_walk_query(size, seed, W.DENSE)
        except A.AsdmError as e:
            if e.code != A.ERR_INVALID:
                raise
            seed += 1
            continue
        q.write(os.path.join(qdir, "q%d.graph" % len(specs)))
        specs.append((size, seed, W.DENSE))
        seed += 1
    return specs


def run_embed(specs, workdir, dpath, cap, jobs):
    """The reference's COLLECT_RESULT build (oracle/_ref/ref_embed) on the
    embed queries: count and the SHA-256 of the sorted embedding dump
    (storeMatches format, matching/join.cpp:1099-1107) where it finished."""
    qdir = os.path.join(workdir, "embed")
    outdir = os.path.join(qdir, "out")
    os.makedirs(outdir, exist_ok=True)
    lst = os.path.join(outdir, "list.txt")
    with open(lst, "w") as fh:
        fh.write("\n".join(os.path.join(qdir, "q%d.graph" % k) for k in range(len(specs))) + "\n")
    r = subprocess.run([REF.replace("ref_local", "ref_embed"), "-d", dpath, "-Q", lst, "-O", outdir, "-T", str(cap),
                        "-J", str(jobs), "-e", "emb"], capture_output=True, text=True, check=True)
    recs = []
    for line in r.stdout.splitlines():
        f = line.split()
        if len(f) < 4 or f[0] != "Q":
            continue
        k = int(f[1])
        size, seed, density = specs[k]
        rec = {"index": k, "seed": seed, "size": size, "density": density, "reference": f[2], "cap_s": cap,
               "wall_s": round(float(f[-1]), 3), "count": None}
        if f[2] == "ok":
            for l in open(os.path.join(outdir, "q%d.out" % k)):
                if l.startswith("Number of matches:"):
                    rec["count"] = int(l.split(":")[1])
            path = os.path.join(outdir, "q%d.emb" % k)
            h = hashlib.sha256()
            with open(path, "rb") as fh:
                for chunk in iter(lambda: fh.read(1 << 20), b""):
                    h.update(chunk)
            rec["emb_sha256"] = h.hexdigest()
            os.remove(path)
        recs.append(rec)
    recs.sort(key=lambda x: x["index"])
    return recs


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cap", type=float, default=60.0)
    ap.add_argument("--jobs", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    ap.add_argument("--workdir", default=os.path.join(ROOT, "_work", "c4ref"))
    ap.add_argument("--parity-only", action="store_true")
    ap.add_argument("--embed-only", action="store_true")
    args = ap.parse_args()
    spec = importlib.util.spec_from_file_location("asdm_specs", os.path.join(ROOT, "asdmatch_b200", "specs.py"))
    S = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(S)
    os.makedirs(args.workdir, exist_ok=True)
    dpath = os.path.join(args.workdir, "data.graph")
    if not os.path.exists(dpath):
        subprocess.run([GEN, "graph"] + S.generator_args(S.C4) + [dpath], check=True)
    old = {}
    if args.parity_only or args.embed_only:
        with open(OUT) as fh:
            old = json.load(fh)
    if old:
        batch = old["queries"]
    else:
        batch = run_reference(S, S.c4_query_specs(), args.workdir, "batch", dpath, args.cap, args.jobs)
    if args.embed_only:
        parity = old["parity"]
    else:
        parity = run_reference(S, S.c4_parity_specs(), args.workdir, "parity", dpath, args.cap, args.jobs)
    embed = run_embed(embed_queries(args.workdir), args.workdir, dpath, args.cap, args.jobs)
    with open(OUT, "w") as fh:
        json.dump({"queries": batch, "parity": parity, "embed": embed,
                   "how": "reference ALL_LEVEL + LOCAL_COUNT build (oracle/_ref/ref_local), one forked process "
                          "per query after one graph load, killed at cap_s; count and the SHA-256 of its CSV "
                          "where it finished"}, fh, indent=0)
    for name, recs in (("queries", batch), ("parity", parity), ("embed", embed)):
        print("c4 golden %s: %d queries, %d finished" % (name, len(recs),
                                                          sum(1 for x in recs if x["count"] is not None)))


if __name__ == "__main__":
    main()
