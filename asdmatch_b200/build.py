"""Builds libasdm_b200.so (sm_100a) and the ASDMatch.out / prepare.out CLIs in-tree.

    python -m asdmatch_b200.build          # or: python asdmatch_b200/build.py

Every CUDA source is compiled with ``-gencode arch=compute_100a,code=sm_100a``;
host sources with g++.  Objects go to asdmatch_b200/_build/, the library to
asdmatch_b200/libasdm_b200.so and the executables to asdmatch_b200/bin/.
Rebuilds only what changed (sources or any header).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libasdm_b200.so")
BIN = os.path.join(PKG, "bin")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc") if os.path.exists(os.path.join(CUDA_HOME, "bin", "nvcc")) else "nvcc"
GENCODE = ["-gencode", "arch=compute_100a,code=sm_100a"]
INCLUDES = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
NVCC_FLAGS = GENCODE + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"] + INCLUDES
CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-march=x86-64-v3", "-Wall", "-Wno-sign-compare",
             "-I", os.path.join(CUDA_HOME, "include")] + INCLUDES


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r.stdout + r.stderr


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(BIN, exist_ok=True)
    hdrs = _headers()
    jobs_list = []
    objs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if _stale(obj, [src] + hdrs):
            if src.endswith(".cu"):
                cmd = [NVCC] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", src, "-o", obj]
            else:
                cmd = ["g++"] + CXX_FLAGS + ["-c", src, "-o", obj]
            jobs_list.append(cmd)
    log = []
    if jobs_list:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for out in ex.map(_run, jobs_list):
                log.append(out)
    if _stale(LIB, objs):
        log.append(_run([NVCC] + GENCODE + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]))
    cli = {"ASDMatch.out": os.path.join(PKG, "cli", "asdmatch_main.cpp"),
           "prepare.out": os.path.join(PKG, "cli", "prepare_main.cpp")}
    for name, src in cli.items():
        if not os.path.exists(src):
            continue
        exe = os.path.join(BIN, name)
        if _stale(exe, [src, LIB] + hdrs):
            log.append(_run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), src,
                             "-L", PKG, "-lasdm_b200", "-Wl,-rpath,$ORIGIN/..", "-o", exe]))
    # the workload generator alone, from its host sources: no CUDA, no library
    gen_src = [os.path.join(PKG, "cli", "gen_main.cpp"), os.path.join(CSRC, "host_graph.cpp")]
    gen = os.path.join(BIN, "asdm_gen.out")
    if all(os.path.exists(x) for x in gen_src) and _stale(gen, gen_src + hdrs):
        log.append(_run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", CSRC] + gen_src +
                        ["-o", gen]))
    text = "".join(log)
    if verbose:
        print(text)
    return text


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
