"""The drop-in executables on the GPU: ASDMatch.out reports, CSV and
embedding dumps against the golden vectors, and prepare.out -> -s."""
import hashlib
import os
import subprocess

import pytest

import asdmatch_b200 as A

pytestmark = pytest.mark.gpu

BIN = A.BIN_DIR


def run(args):
    r = subprocess.run([os.path.join(BIN, args[0])] + args[1:], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return r.stdout


def matches(out):
    return int([l for l in out.splitlines() if l.startswith("Number of matches:")][0].split(":")[1])


def sha(path):
    return hashlib.sha256(open(path, "rb").read()).hexdigest()


def test_asdmatch_out_counts_csv_and_embeddings(golden, c0_files, tmp_path):
    _, dpath, _, qpaths = c0_files
    done = 0
    for rec in golden["sets"]["c0"]:
        if "csv_sha" not in rec or done >= 6:
            continue
        csv, emb, rep = str(tmp_path / "l.csv"), str(tmp_path / "e.txt"), str(tmp_path / "r.txt")
        run(["ASDMatch.out", "-q", qpaths[rec["index"]], "-d", dpath, "-c", csv, "-e", emb, "-r", rep])
        report = open(rep).read()
        assert matches(report) == rec["count"]
        for key in ("Filtering time (s):", "Planning Time:", "Execution Time:", "Number of intersections:"):
            assert key in report
        assert sha(csv) == rec["csv_sha"] and sha(emb) == rec["emb_sha"]
        done += 1
    assert done == 6


def test_prepare_then_plan_from_card(golden, c0d_files, tmp_path):
    _, dpath, by_size = c0d_files
    for rec in golden["sets"]["c0d"][40:46]:
        qpath = by_size[rec["size"]][1][rec["index"]]
        card = str(tmp_path / "q.card")
        run(["prepare.out", "-q", qpath, "-d", dpath, "-s", card])
        info = A.Card(card).info()
        assert info["entries"] > 0
        out = run(["ASDMatch.out", "-q", qpath, "-d", dpath, "-s", card])
        assert "dp time:" in out
        assert matches(out) == rec["count"]


def test_missing_file_message(tmp_path):
    r = subprocess.run([os.path.join(BIN, "ASDMatch.out"), "-q", str(tmp_path / "x"), "-d", str(tmp_path / "y")],
                       capture_output=True, text=True, timeout=60)
    assert "Can not open file" in r.stdout and r.returncode != 0
