"""Pin the float64 oracle to the reference's own code.

geometry_ref.npz holds outputs of the reference orbit.cu / bounds.cu compiled
as host C++ (tests/golden/make_geometry_golden.py).  The oracle restates the
same operations in the same order, so it must agree to the last bit up to
libm differences (sin/cos/atan may differ by an ulp between glibc and NumPy).
When oracle/_ref/libref_geom.so is present the comparison also runs live.
"""
import ctypes
import os

import numpy as np
import pytest

from oracle import geometry as og

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "geometry_ref.npz")
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libref_geom.so")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLD)


def test_llh2xyz_and_back(g):
    np.testing.assert_allclose(og.llh2xyz(g["llh"]), g["xyz"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(og.xyz2llh(g["xyz"]), g["llh_back"], rtol=0, atol=1e-9)


def test_intp_orbit(g):
    sx, sv = og.intp_orbit(g["tt"], g["xx"], g["vv"], g["t"])
    np.testing.assert_allclose(sx, g["satx"], rtol=0, atol=1e-7)
    np.testing.assert_allclose(sv, g["satv"], rtol=0, atol=1e-9)


def test_orbitrangetime(g):
    xm, vm = og.intp_orbit(g["tt"], g["xx"], g["vv"], np.float64(g["tmid"]))
    tl, dr, it = og.orbitrangetime(g["tt"], g["xx"], g["vv"], g["ground_xyz"], float(g["tmid"]), xm, vm)
    np.testing.assert_allclose(tl, g["tline"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(dr, g["dr"], rtol=0, atol=1e-6)
    assert it.max() <= 51


def test_bounds(g):
    for c, want in zip(g["bound_cases"], g["bounds"]):
        got = og.bounds(*c, g["tt"], g["xx"], g["vv"])
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-11)


@pytest.mark.skipif(not os.path.exists(LIB), reason="reference geometry library not built")
def test_live_reference_bit_exact():
    lib = ctypes.CDLL(LIB)
    P = ctypes.POINTER(ctypes.c_double)
    rng = np.random.default_rng(1)
    from sentinel_gpu_processor_b200 import synth
    tt, xx, vv = [np.ascontiguousarray(a) for a in synth.make_orbit()]
    t = np.ascontiguousarray(rng.uniform(tt[0], tt[-1], 500))
    sx, sv = np.zeros((500, 3)), np.zeros((500, 3))
    lib.ref_intp_orbit(ctypes.c_long(len(tt)), tt.ctypes.data_as(P), xx.ctypes.data_as(P), vv.ctypes.data_as(P),
                       t.ctypes.data_as(P), ctypes.c_long(500), sx.ctypes.data_as(P), sv.ctypes.data_as(P))
    ox, ov = og.intp_orbit(tt, xx, vv, t)
    np.testing.assert_array_equal(ox, sx)
    np.testing.assert_array_equal(ov, sv)
