"""Generate ``geometry_ref.npz``: outputs of the reference's own geometry code
(csrc/src/orbit.cu, csrc/src/bounds.cu compiled as host C++ into
oracle/_ref/libref_geom.so by oracle/build_ref.py) on seeded inputs.

Run from the repository root: ``python tests/golden/make_geometry_golden.py``.
The fixture pins oracle/geometry.py (tests/test_oracle_pins.py) without the
reference being present.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from sentinel_gpu_processor_b200 import synth  # noqa: E402

LIB = os.path.join(ROOT, "oracle", "_ref", "libref_geom.so")
P = ctypes.POINTER(ctypes.c_double)


def ptr(a):
    return a.ctypes.data_as(P)


def main():
    lib = ctypes.CDLL(LIB)
    rng = np.random.default_rng(20261203)
    tt, xx, vv = [np.ascontiguousarray(a) for a in synth.make_orbit()]
    n = 400
    llh = np.ascontiguousarray(np.stack([rng.uniform(33, 38, n), rng.uniform(12, 16, n),
                                         rng.uniform(-100, 3000, n)], -1))
    xyz = np.zeros_like(llh)
    lib.ref_llh2xyz(ptr(llh), ptr(xyz), ctypes.c_long(n))
    llh_back = np.zeros_like(llh)
    lib.ref_xyz2llh(ptr(xyz), ptr(llh_back), ctypes.c_long(n))
    t = np.ascontiguousarray(rng.uniform(tt[0] - 5, tt[-1] + 5, n))
    sx, sv = np.zeros((n, 3)), np.zeros((n, 3))
    lib.ref_intp_orbit(ctypes.c_long(len(tt)), ptr(tt), ptr(xx), ptr(vv), ptr(t), ctypes.c_long(n), ptr(sx), ptr(sv))
    # ground points in the swath of the synthetic orbit
    g = np.ascontiguousarray(np.stack([rng.uniform(35.4, 36.0, n), rng.uniform(13.8, 14.6, n),
                                       rng.uniform(0, 3000, n)], -1))
    gx = np.zeros_like(g)
    lib.ref_llh2xyz(ptr(g), ptr(gx), ctypes.c_long(n))
    tmid = float(tt[5])
    xm, vm = np.zeros((1, 3)), np.zeros((1, 3))
    lib.ref_intp_orbit(ctypes.c_long(len(tt)), ptr(tt), ptr(xx), ptr(vv), ptr(np.array([tmid])), ctypes.c_long(1),
                       ptr(xm), ptr(vm))
    tl, dr = np.zeros(n), np.zeros((n, 3))
    lib.ref_orbitrangetime(ctypes.c_long(len(tt)), ptr(tt), ptr(xx), ptr(vv), ptr(gx), ctypes.c_long(n),
                           ctypes.c_double(tmid), ptr(np.ascontiguousarray(xm[0])), ptr(np.ascontiguousarray(vm[0])),
                           ptr(tl), ptr(dr))
    bcases = np.array([[50048.0, 50051.0, 8.0e5, 8.49e5, -100.0, 3000.0],
                       [50040.0, 50043.1, 8.45e5, 9.0e5, -100.0, 9000.0],
                       [50055.5, 50058.4, 8.9e5, 9.5e5, 0.0, 1500.0]])
    bout = np.zeros((len(bcases), 4))
    for i, c in enumerate(bcases):
        o = np.zeros(4)
        lib.ref_bounds(*[ctypes.c_double(v) for v in c], ptr(tt), ptr(xx), ptr(vv), ctypes.c_long(len(tt)), ptr(o))
        bout[i] = o
    np.savez_compressed(os.path.join(os.path.dirname(os.path.abspath(__file__)), "geometry_ref.npz"),
                        tt=tt, xx=xx, vv=vv, llh=llh, xyz=xyz, llh_back=llh_back, t=t, satx=sx, satv=sv,
                        ground_llh=g, ground_xyz=gx, tmid=tmid, tline=tl, dr=dr, bound_cases=bcases,
                        bounds=bout)
    print("wrote geometry_ref.npz")


if __name__ == "__main__":
    main()
