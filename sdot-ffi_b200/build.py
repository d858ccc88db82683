"""Builds libsdot_b200.so in-tree: every .cu of csrc/ for sm_100a (nvcc), linked as one shared library.

    python sdot-ffi_b200/build.py [--jobs N] [--debug]

The library lands in sdot-ffi_b200/sdot/_lib/ next to the Python package that loads it.
"""
import argparse
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "sdot", "_lib")
LIB = os.path.join(OUT_DIR, "libsdot_b200.so")
BUILD = os.path.join(HERE, "_build")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    hs.append(os.path.join(HERE, "..", "include", "sdot_b200.h"))
    return hs


def compile_one(src, debug, verbose):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest = max(os.path.getmtime(h) for h in headers() + [src])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest:
        return obj
    flags = ["-O3", "-lineinfo"] if not debug else ["-O0", "-g", "-G"]
    cmd = ["nvcc", *ARCH, *flags, "-std=c++17", "-Xcompiler", "-fPIC,-O3", "-Xptxas", "-v" if verbose else "-O3",
           "-I", os.path.join(HERE, "..", "include"), "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"nvcc failed on {src}")
    if verbose:
        sys.stderr.write(r.stderr)
    return obj


def build(jobs=8, debug=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(OUT_DIR, exist_ok=True)
    with concurrent.futures.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda s: compile_one(s, debug, verbose), sources()))
    newest = max(os.path.getmtime(o) for o in objs)
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = ["nvcc", *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.debug, a.verbose))
