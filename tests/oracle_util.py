"""Test-side access to the CPU oracle (oracle/asdm_oracle.cpp) and, when it was
built here, to the reference build in oracle/_ref.  Checker only: nothing in
the product imports this module."""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import subprocess

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_LIB = os.path.join(ROOT, "oracle", "_build", "liboracle_asdm.so")
ORACLE_BIN = os.path.join(ROOT, "oracle", "_build", "asdm_oracle")
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

MODE_COUNT, MODE_LOCAL, MODE_EMBED = 0, 1, 2


def reference_tree():
    """The reference source tree oracle/ref.mk builds from (that recipe holds
    the location; $ASDM_REFERENCE_DIR overrides it), or None when absent."""
    try:
        r = subprocess.run(["make", "-s", "-f", "oracle/ref.mk", "refdir"], cwd=ROOT, capture_output=True,
                           text=True, timeout=30)
    except (OSError, subprocess.TimeoutExpired):
        return None
    d = r.stdout.strip()
    return d if r.returncode == 0 and d and os.path.isdir(d) else None


def reference_file(*parts):
    """A file of the reference tree (e.g. its yeast dataset), or None."""
    d = reference_tree()
    if d is None:
        return None
    p = os.path.join(d, *parts)
    return p if os.path.exists(p) else None


def build_oracle():
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < os.path.getmtime(
            os.path.join(ROOT, "oracle", "asdm_oracle.cpp")):
        subprocess.run(["make", "-s", "-f", "oracle/Makefile"], cwd=ROOT, check=True)


_lib = None


def _oracle():
    global _lib
    if _lib is None:
        build_oracle()
        _lib = C.CDLL(ORACLE_LIB)
        _lib.orc_run.restype = C.c_int
        _lib.orc_run.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32),
                                 C.c_char_p, C.c_char_p, C.c_char_p]
    return _lib


def oracle_run(qpath, dpath, mode=MODE_COUNT, csv=None, emb=None, cs=None):
    """Returns (count, flags); writes the CSV / embedding dump / candidate-space dump when paths are given."""
    c = C.c_uint64()
    f = C.c_uint32()
    enc = lambda p: (p or "").encode()
    rc = _oracle().orc_run(qpath.encode(), dpath.encode(), mode, C.byref(c), C.byref(f), enc(csv), enc(emb), enc(cs))
    if rc != 0:
        raise RuntimeError("oracle failed with %d" % rc)
    return c.value, f.value


def sha256_file(path):
    h = hashlib.sha256()
    with open(path, "rb") as fh:
        for chunk in iter(lambda: fh.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def sha256_bytes(b):
    return hashlib.sha256(b).hexdigest()


def ref_available():
    return all(os.path.exists(os.path.join(REF_DIR, n)) for n in ("ref_count", "ref_local", "ref_embed"))


def ref_run(variant, qpath, dpath, csv=None, emb=None, cs=None, timeout=300):
    """Runs a reference build; returns its 'Number of matches' (None on an empty candidate space)."""
    cmd = [os.path.join(REF_DIR, variant), "-q", qpath, "-d", dpath]
    if csv:
        cmd += ["-c", csv]
    if emb:
        cmd += ["-e", emb]
    if cs:
        cmd += ["-w", cs]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("reference failed: %s\n%s" % (r.stdout, r.stderr))
    for line in r.stdout.splitlines():
        if line.startswith("Number of matches:"):
            return int(line.split(":")[1])
    raise RuntimeError("no count in reference output:\n" + r.stdout)
