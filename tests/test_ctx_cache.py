"""Keying of the device address that s1b_goldstein_noalloc caches.

The address of a module's device array belongs to a CUDA context, so the
cache is keyed on the context handle and the context's unique id.  The
cache (csrc/s1b_ctx_cache.h) is host code; this test compiles a small
check program against it with the host compiler and runs it on the CPU,
with stand-in handles for contexts.
"""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "sentinel_gpu_processor_b200", "csrc")


def test_context_keyed_cache(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path / "ctx_cache_check")
    subprocess.run([gxx, "-std=c++17", "-O1", "-I" + CSRC, os.path.join(HERE, "native", "ctx_cache_check.cpp"),
                    "-o", exe, "-pthread"], check=True)
    r = subprocess.run([exe], stdout=subprocess.PIPE, text=True)
    assert r.returncode == 0, r.stdout
    assert "ctx cache ok" in r.stdout
