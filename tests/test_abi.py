"""The C ABI: libs1b.so loads without a GPU and exports every function that
include/s1b.h declares; struct layouts match the ctypes mirror."""
import ctypes
import os
import re

from sentinel_gpu_processor_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names |= set(re.findall(r"\b(s1b_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    decl = declared_functions()
    assert len(decl) >= 15
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declarations():
    assert set(declared_functions()) <= set(_lib.exported_symbols())


def test_struct_layout_and_host_calls():
    lib = _lib.load()
    assert lib.s1b_sizeof_burst_plan() == ctypes.sizeof(_lib.BurstPlan)
    assert lib.s1b_sizeof_orbit_poly() == ctypes.sizeof(_lib.OrbitPoly)
    assert lib.s1b_version() >= 100
    assert _lib.status_string(0) == "ok"
    # a device call without a GPU (or with bad args) reports a status, never exits
    st = lib.s1b_deramp(None, None, None, None)
    assert st == _lib.S1B_ERR_INVALID_ARGUMENT


def test_frame_structs_and_argument_checks():
    assert ctypes.sizeof(_lib.FramePair) == 72
    assert ctypes.sizeof(_lib.FrameSizes) == 32
    lib = _lib.load()
    h = ctypes.c_void_p()
    st = lib.s1b_frame_create(None, 0, None, None, 0, 1, 1, 32, 0.5, 0, ctypes.byref(h))
    assert st == _lib.S1B_ERR_INVALID_ARGUMENT and not h.value
    assert lib.s1b_frame_sizes(None, None) == _lib.S1B_ERR_INVALID_ARGUMENT
    lib.s1b_frame_destroy(None)  # accepts NULL
