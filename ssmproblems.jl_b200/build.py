"""Build libgfb200.so from csrc/*.cu with nvcc for sm_100a (B200).

Usage: python ssmproblems.jl_b200/build.py [--force] [--jobs N]

Objects go to ssmproblems.jl_b200/_build/, the shared library to
ssmproblems.jl_b200/lib/libgfb200.so (in-tree, so it travels with the source).
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libgfb200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "--use_fast_math",
         "-I", INCLUDE]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.hpp")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def _deps(dep_file):
    """Headers listed in an nvcc -MD dependency file (None if absent)."""
    if not os.path.exists(dep_file):
        return None
    text = open(dep_file).read().replace("\\\n", " ")
    parts = text.split(":", 1)
    return parts[1].split() if len(parts) == 2 else None


def _stale(obj, src, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    if m < os.path.getmtime(src):
        return True
    deps = _deps(obj[:-2] + ".d")
    if deps is None:
        return m < hdr_mtime
    return any(not os.path.exists(d) or m < os.path.getmtime(d) for d in deps)


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or _stale(o, s, hdr_mtime):
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        t0 = time.time()
        cmd = [NVCC] + ARCH + FLAGS + ["-MD", "-MF", o[:-2] + ".d", "-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {s}:\n{r.stdout}\n{r.stderr}")
        # date the object at the compile's start: a source or header edited while
        # nvcc ran then still counts as newer, and the next build recompiles it
        os.utime(o, (t0, t0))
        if verbose:
            print(f"compiled {os.path.basename(s)}", flush=True)
        return o

    if todo:
        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(compile_one, todo))
    if todo or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=True))
    sys.exit(0)
