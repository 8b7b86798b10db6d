"""Build the reference checker into ``oracle/_ref/`` from the reference sources.

Test infrastructure only.  Nothing is copied: the compilers read the sources
where they lie (``/root/reference/csrc``) and write only into ``oracle/_ref``
(git-ignored; it travels to the GPU box with the working tree).

Outputs
  * ``libref_geom.so`` -- ``csrc/src/orbit.cu`` and ``csrc/src/bounds.cu``
    compiled as host C++ (``-D__host__= -D__device__=``) plus the extern "C"
    wrapper ``oracle/ref_shim/ref_geom_shim.cpp``.  Runs on any CPU and pins
    the float64 geometry oracle to the reference's own code.
  * ``bin/geo2rdr``, ``bin/crossmul_daemon``, ``bin/crossmul``,
    ``bin/goldstein`` -- the reference executables built by nvcc for sm_100a
    with the source lists of ``csrc/CMakeLists.txt:67-71``.  geo2rdr links the
    system ``libsqlite3.so.0`` through the prototype-only header in
    ``oracle/ref_shim/``.  They run on the B200 box only.
  * ``bin/kbench_chain``, ``bin/kbench_goldstein`` -- kernel-only timing
    harnesses (``oracle/ref_shim/kbench_*.cu``) that include the reference's
    geo2rdr.cu / goldstein.cu and time its kernels on device-resident inputs.

Usage: ``python oracle/build_ref.py [--reference DIR] [--geom-only]``.  The
reference source tree is the argument, else the ``S1B_REFERENCE_DIR``
environment variable, else the recipe's default location; when none of them
holds the sources nothing is built (a prebuilt ``oracle/_ref`` is kept).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SQLITE_SO = "/usr/lib/x86_64-linux-gnu/libsqlite3.so.0"
DEFAULT_REFERENCE = "/root/reference"


def reference_dir(reference=None):
    return reference or os.environ.get("S1B_REFERENCE_DIR") or DEFAULT_REFERENCE


def _run(cmd, log):
    log.write("$ " + " ".join(cmd) + "\n")
    log.flush()
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    log.write(r.stdout)
    log.flush()
    if r.returncode != 0:
        raise RuntimeError(f"reference build step failed: {' '.join(cmd[:3])} ... (see {log.name})")


def build(reference=None, geom_only=False, quiet=True):
    reference = reference_dir(reference)
    src = os.path.join(reference, "csrc", "src")
    inc = os.path.join(reference, "csrc", "include")
    if not os.path.isdir(src):
        return False
    os.makedirs(os.path.join(OUT, "bin"), exist_ok=True)
    with open(os.path.join(OUT, "build.log"), "w") as log:
        gxx = shutil.which("g++") or "g++"
        _run([gxx, "-O2", "-fPIC", "-shared", "-std=c++14", "-D__host__=", "-D__device__=",
              "-I" + inc, "-x", "c++", os.path.join(src, "orbit.cu"), os.path.join(src, "bounds.cu"),
              "-x", "c++", os.path.join(HERE, "ref_shim", "ref_geom_shim.cpp"),
              "-o", os.path.join(OUT, "libref_geom.so")], log)
        if geom_only:
            return True
        nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
        common = [nvcc, "-O3", "-std=c++17", *ARCH, "-I" + inc, "-I" + os.path.join(HERE, "ref_shim")]
        _run(common + ["-rdc=true", os.path.join(src, "geo2rdr.cu"), os.path.join(src, "sql_mod.cpp"),
                       os.path.join(src, "orbit.cu"), os.path.join(src, "sario.cu"),
                       os.path.join(src, "bounds.cu"), "-Xlinker", SQLITE_SO,
                       "-o", os.path.join(OUT, "bin", "geo2rdr")], log)
        _run(common + [os.path.join(src, "crossmul_daemon.cu"), os.path.join(src, "sario.cu"),
                       "-o", os.path.join(OUT, "bin", "crossmul_daemon")], log)
        _run(common + [os.path.join(src, "crossmul.cu"), os.path.join(src, "sario.cu"),
                       "-o", os.path.join(OUT, "bin", "crossmul")], log)
        _run(common + [os.path.join(src, "goldstein.cu"), "-lcufft",
                       "-o", os.path.join(OUT, "bin", "goldstein")], log)
        # kernel-only timing harnesses: the reference's kernels on device-resident
        # inputs (the harness sources include the reference files where they lie)
        shim = os.path.join(HERE, "ref_shim")
        _run(common + ["-rdc=true", "-I" + src, os.path.join(shim, "kbench_chain.cu"),
                       os.path.join(src, "sql_mod.cpp"), os.path.join(src, "orbit.cu"), os.path.join(src, "sario.cu"),
                       os.path.join(src, "bounds.cu"), "-Xlinker", SQLITE_SO,
                       "-o", os.path.join(OUT, "bin", "kbench_chain")], log)
        _run(common + ["-I" + src, os.path.join(shim, "kbench_goldstein.cu"), "-lcufft",
                       "-o", os.path.join(OUT, "bin", "kbench_goldstein")], log)
    return True


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    ap.add_argument("--geom-only", action="store_true")
    a = ap.parse_args()
    ok = build(a.reference, a.geom_only)
    print("built" if ok else "reference sources not found; nothing built")
    sys.exit(0)
