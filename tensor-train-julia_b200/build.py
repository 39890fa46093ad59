"""Build libttcuda.so (sm_100a) in-tree with nvcc.

    python tensor-train-julia_b200/build.py [--jobs N] [--debug]

The shared library lands next to the Python host package (ttcuda/libttcuda.so), so a
Julia ccall or the Python ctypes loader finds it without installation.  Object files go
to _build/ beside this script.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "ttcuda", "libttcuda.so")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(jobs: int = 8, debug: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "ttcuda.h"))
    flags = ARCH + ["-std=c++17", "-Xcompiler", "-fPIC", "-lineinfo", "-I", INCLUDE,
                    "-O0" if debug else "-O3", "--expt-relaxed-constexpr"]
    if debug:
        flags += ["-DTTC_DEBUG"]
    if ptxas_v:
        flags += ["-Xptxas", "-v"]
    objs, todo = [], []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if newer(obj, [src] + headers) or ptxas_v:
            todo.append((src, obj))

    def compile_one(item):
        src, obj = item
        cmd = [nvcc()] + flags + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
        return src, r.stderr

    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for src, err in ex.map(compile_one, todo):
            if ptxas_v and err:
                print(f"== {os.path.basename(src)}\n{err}")
    if todo or not os.path.exists(OUT):
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", OUT] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.jobs, a.debug, a.verbose, a.ptxas_v))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)
