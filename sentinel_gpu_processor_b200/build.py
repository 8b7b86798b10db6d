"""Build ``libs1b.so`` (the s1b C ABI) in-tree for sm_100a with nvcc.

Usage: ``python -m sentinel_gpu_processor_b200.build [--force] [--verbose-ptxas]``.
Objects go to ``sentinel_gpu_processor_b200/_build/``; the shared library to
``sentinel_gpu_processor_b200/libs1b.so``.  Sources are rebuilt when they or
any header are newer than their object.
"""
from __future__ import annotations

import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libs1b.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# per-source flags: the device burst geometry rounds FP64 operation by
# operation like the host planner (no FMA contraction)
EXTRA_FLAGS = {"k_plan.cu": ["-fmad=false"]}


def _nvcc():
    p = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(p):
        raise RuntimeError("nvcc not found")
    return p


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
                  + glob.glob(os.path.join(INCLUDE, "*.h")))


def build(force=False, verbose_ptxas=False, quiet=False):
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    hdr_mtime = max((os.path.getmtime(h) for h in headers()), default=0.0)
    objs = []
    flags = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
             *ARCH]
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_mtime):
            continue
        cmd = [nvcc, *flags, *EXTRA_FLAGS.get(os.path.basename(src), []), "-c", src, "-o", obj]
        if verbose_ptxas and src.endswith(".cu"):
            cmd[1:1] = ["-Xptxas", "-v"]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0 or (verbose_ptxas and not quiet):
            sys.stderr.write(r.stdout)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}")
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [nvcc, *ARCH, "-shared", "-o", LIB, *objs]
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout)
            raise RuntimeError("link of libs1b.so failed")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose-ptxas", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose_ptxas=a.verbose_ptxas))
