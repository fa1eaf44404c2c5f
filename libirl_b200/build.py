"""Builds libirl_b200/libirl_b200.so in place.

Host C (libirl_b200/csrc/host/*.c) is compiled by gcc with libirl's
arithmetic model (x86-64 SSE, no FP contraction); the CUDA sources
(libirl_b200/csrc/cuda/*.cu) by nvcc for sm_100a only.  Objects go to
libirl_b200/_build/; a source is recompiled when it or any header is newer
than its object.

    python -m libirl_b200.build [-j N] [--force]
"""
from __future__ import annotations

import argparse
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJ = os.path.join(PKG, "_build")
SO = os.path.join(PKG, "libirl_b200.so")
INCLUDE = os.path.join(ROOT, "include")
NVCC = os.environ.get("NVCC", "nvcc")
CC = os.environ.get("CC", "gcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-ffp-contract=off", f"-I{INCLUDE}"]
CC_FLAGS = ["-O2", "-std=gnu99", "-fPIC", "-pthread", "-ffp-contract=off", "-Wall",
            "-Wno-unused-function", f"-I{INCLUDE}"]


def _headers():
    return (glob.glob(os.path.join(CSRC, "**", "*.h"), recursive=True)
            + glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True)
            + glob.glob(os.path.join(INCLUDE, "*.h")))


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or hdr_mtime > t


def _compile(job):
    src, obj = job
    if src.endswith(".cu"):
        cmd = [NVCC] + NVCC_FLAGS + ["-c", src, "-o", obj]
    else:
        cmd = [CC] + CC_FLAGS + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return obj


def build(jobs: int | None = None, force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "host", "*.c")) + glob.glob(os.path.join(CSRC, "cuda", "*.cu")))
    hdr_mtime = max([os.path.getmtime(h) for h in _headers()] + [0])
    todo, objs = [], []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(s, o, hdr_mtime):
            todo.append((s, o))
    if todo:
        if verbose:
            print(f"compiling {len(todo)} file(s)", file=sys.stderr)
        with ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
            list(ex.map(_compile, todo))
    if todo or not os.path.exists(SO) or any(os.path.getmtime(o) > os.path.getmtime(SO) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", SO] + objs + ["-lm", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return SO


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.j, a.force, verbose=True))
