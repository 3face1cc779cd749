"""Reference results for the config-4 queries (tests/golden/c4_batch.json).

    python tests/golden/make_c4_golden.py [--cap S] [--jobs J]

Config 4 is local subgraph counting: the Chung-Lu graph N=1.0M, M=10M,
exponent 2.3, 32 labels Zipf(1.0), and 50 random-walk queries of 10 vertices
(seeds 90,000 + i).  This script writes them with the host-only generator
(asdmatch_b200/bin/asdm_gen.out) and runs the reference's ALL_LEVEL +
LOCAL_COUNT build (oracle/_ref/ref_local) on each query in its own forked
process after one graph load, killed at the cap.  Where the reference
finished it records the count and the SHA-256 of the |Vg| x |Vq| CSV it wrote
(main.cpp:135-146); otherwise that it did not finish.
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--cap", type=float, default=60.0)
    ap.add_argument("--jobs", type=int, default=max(1, (os.cpu_count() or 2) - 2))
    ap.add_argument("--workdir", default=os.path.join(ROOT, "_work", "c4ref"))
    args = ap.parse_args()
    spec = importlib.util.spec_from_file_location("asdm_specs", os.path.join(ROOT, "asdmatch_b200", "specs.py"))
    S = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(S)
    os.makedirs(args.workdir, exist_ok=True)
    dpath = os.path.join(args.workdir, "data.graph")
    if not os.path.exists(dpath):
        subprocess.run([GEN, "graph"] + S.generator_args(S.C4) + [dpath], check=True)
    specs = S.c4_query_specs()
    gl = os.path.join(args.workdir, "gen.txt")
    with open(gl, "w") as fh:
        for k, (size, seed, density) in enumerate(specs):
            fh.write("%d %d %d q%d.graph\n" % (size, seed, density, k))
    subprocess.run([GEN, "queries"] + S.generator_args(S.C4) + [gl, args.workdir], check=True)
    outdir = os.path.join(args.workdir, "out")
    os.makedirs(outdir, exist_ok=True)
    lst = os.path.join(outdir, "list.txt")
    with open(lst, "w") as fh:
        fh.write("\n".join(os.path.join(args.workdir, "q%d.graph" % k) for k in range(len(specs))) + "\n")
    r = subprocess.run([REF, "-d", dpath, "-Q", lst, "-O", outdir, "-T", str(args.cap), "-J", str(args.jobs),
                        "-c", "csv"], capture_output=True, text=True, check=True)
    recs = []
    for line in r.stdout.splitlines():
        f = line.split()
        if len(f) < 4 or f[0] != "Q":
            continue
        k = int(f[1])
        size, seed, density = specs[k]
        rec = {"index": k, "seed": seed, "size": size, "reference": f[2], "cap_s": args.cap,
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
    with open(OUT, "w") as fh:
        json.dump({"queries": recs, "how": "reference ALL_LEVEL + LOCAL_COUNT build (oracle/_ref/ref_local), one "
                                           "forked process per query after one graph load, killed at cap_s; "
                                           "count and the SHA-256 of its CSV where it finished"}, fh, indent=0)
    print("c4 golden: %d queries, %d finished" % (len(recs), sum(1 for x in recs if x["count"] is not None)))


if __name__ == "__main__":
    main()
