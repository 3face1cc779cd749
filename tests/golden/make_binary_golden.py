"""Digests of the reference's binary graph cache (Graph::writeToStream,
relation/graph.cpp:316-332) for the seeded config-0 graphs, written by the
reference build in oracle/_ref (`ref_count -b`).  Output:
tests/golden/binary_graph.json.  Run from the repository root after building
oracle/_ref."""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from asdmatch_b200 import workloads as W  # noqa: E402


def main():
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, spec in (("c0", W.C0), ("c0d", W.C0D)):
            g = W.graph(spec)
            dpath = os.path.join(tmp, name + ".graph")
            g.write(dpath)
            bpath = os.path.join(tmp, name + ".bin")
            subprocess.run([os.path.join(ROOT, "oracle", "_ref", "ref_count"), "-q", dpath, "-d", dpath, "-b", bpath],
                           check=True, capture_output=True)
            with open(bpath, "rb") as fh:
                data = fh.read()
            out[name] = {"spec": spec, "bytes": len(data), "sha256": hashlib.sha256(data).hexdigest()}
    with open(os.path.join(HERE, "binary_graph.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
