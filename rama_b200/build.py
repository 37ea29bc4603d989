"""Builds the in-tree native artefacts for sm_100a.

    python -m rama_b200.build [--force]

* rama_b200/librama_b200.so   -- the CUDA solver behind include/rama_b200.h
* rama_b200/bin/rama_text_input -- the command-line front end

A target is rebuilt when any of its sources is newer than it.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "librama_b200.so")
CLI = os.path.join(HERE, "bin", "rama_text_input")
NVCC = os.environ.get("NVCC", "nvcc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-std=c++17", "-O3", "-lineinfo",
    # strict IEEE arithmetic so that results match the CPU oracle bit for bit
    "-fmad=false",
    "--expt-relaxed-constexpr", "--extended-lambda",
    "-Xcompiler", "-fPIC",
]
# RAMA_SPLIT_COMPILE=1 also splits the optimisation of each unit over the
# host cores.  Development builds only: the C2 solve measured about 2 % slower
# built that way.
if os.environ.get("RAMA_SPLIT_COMPILE") == "1":
    NVCC_FLAGS.append("--split-compile=0")


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_lib(force=False, verbose=False):
    """Compiles every stale csrc/*.cu to an object (all in parallel: each
    kernel has a translation unit of its own) and links the .so.  An object
    is stale when its .cu, any header or the C ABI header is newer."""
    headers = glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(INCLUDE, "rama_b200.h")]
    units = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
    objdir = os.path.join(HERE, "_build")
    objects = [os.path.join(objdir, os.path.basename(u)[:-3] + ".o") for u in units]
    if not force and not _stale(LIB, units + headers) and all(os.path.exists(o) for o in objects):
        return LIB
    os.makedirs(objdir, exist_ok=True)
    # Outputs are stamped with the time their compile started, so that a
    # source edited while the build runs stays newer than its object.
    started = time.time()
    procs, objs = [], []
    for u in units:
        o = os.path.join(objdir, os.path.basename(u)[:-3] + ".o")
        objs.append(o)
        if not force and not _stale(o, [u] + headers):
            continue
        cmd = [NVCC, *NVCC_FLAGS, "-c", "-o", o, u]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        procs.append((subprocess.Popen(cmd), o))
    if any(p.wait() != 0 for p, _ in procs):
        raise RuntimeError("nvcc failed")
    for _, o in procs:
        os.utime(o, (started, started))
    subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp", *objs],
                   check=True)
    os.utime(LIB + ".tmp", (started, started))
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_cli(force=False):
    src = os.path.join(HERE, "cli", "rama_text_input.cpp")
    hdrs = glob.glob(os.path.join(INCLUDE, "*.h"))
    if not force and not _stale(CLI, [src, LIB, *hdrs]):
        return CLI
    os.makedirs(os.path.dirname(CLI), exist_ok=True)
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", INCLUDE, "-o", CLI, src, "-L", HERE, "-l:librama_b200.so",
                    "-Wl,-rpath,$ORIGIN/.."], check=True)
    return CLI


def build(force=False):
    build_lib(force)
    build_cli(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("built", LIB, "and", CLI)
