"""Builds libdsss.so (all CUDA kernels and host code, sm_100a) in this directory.

Every source compiles to its own object in parallel (one process per source),
then one link makes the shared library.

Usage: python build.py [--force]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "libdsss.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3"]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    return ([os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
            + [os.path.join(HERE, "..", "include", "dsss.h")])


def deps():
    return sources() + headers()


def up_to_date():
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in deps())


def _obj(src):
    return os.path.join(OBJ, os.path.basename(src) + ".o")


def _compile(src, force, hdr_time, verbose):
    obj = _obj(src)
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time)):
        return
    cmd = [NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj + ".tmp"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(obj + ".tmp", obj)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return OUT
    os.makedirs(OBJ, exist_ok=True)
    hdr_time = max(os.path.getmtime(h) for h in headers())
    srcs = sources()
    jobs = max(1, min(len(srcs), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        for f in [ex.submit(_compile, s, force, hdr_time, verbose) for s in srcs]:
            f.result()
    cmd = [NVCC] + ARCH + ["-shared"] + [_obj(s) for s in srcs] + ["-o", OUT + ".tmp", "-lpthread"]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
