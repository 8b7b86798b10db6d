"""Host-side planning: build the C records of ``include/s1b.h`` from Python
objects and call the library's planners (no GPU needed)."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def _as_c(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def c_orbit(tt, xx, vv):
    tt, pt = _as_c(tt)
    xx, px = _as_c(np.asarray(xx).reshape(-1))
    vv, pv = _as_c(np.asarray(vv).reshape(-1))
    return _lib.Orbit(len(tt), pt, px, pv), (tt, xx, vv)


def c_poly_table(tab):
    tab = np.asarray(tab, dtype=np.float64).reshape(-1, 5)
    cols = [np.ascontiguousarray(tab[:, k]) for k in range(5)]
    ptrs = [c.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for c in cols]
    return _lib.PolyTable(len(tab), *ptrs), cols


def c_radar(r):
    return _lib.Radar(int(r.samples_per_burst), int(r.lines_per_burst), float(r.prf), float(r.wvl),
                      float(r.hmin), float(r.hmax), float(r.range_sampling_rate), float(r.slant_range_time),
                      float(r.azimuth_steering_rate), float(r.azimuth_time_interval), float(r.radar_frequency))


def c_burst(b):
    return _lib.Burst(float(b.azimuth_time), int(b.first_valid_line), int(b.last_valid_line),
                      int(b.first_valid_sample), int(b.last_valid_sample))


def c_rsc(r):
    return _lib.Rsc(int(r.nlat), int(r.nlon), float(r.latmax), float(r.lonmin), float(r.dlat), float(r.dlon))


def orbit_poly(tt, xx, vv) -> _lib.OrbitPoly:
    lib = _lib.load()
    orb, keep = c_orbit(tt, xx, vv)
    out = _lib.OrbitPoly()
    _lib.check(lib.s1b_orbit_poly(ctypes.byref(orb), ctypes.byref(out)), "s1b_orbit_poly")
    return out


def orbit_eval(poly: _lib.OrbitPoly, t):
    """Host evaluation of the orbit polynomials: (satx [n,3], satv [n,3])."""
    lib = _lib.load()
    t, pt = _as_c(np.atleast_1d(t))
    x = np.zeros((len(t), 3))
    v = np.zeros((len(t), 3))
    _lib.check(lib.s1b_orbit_eval_host(ctypes.byref(poly), pt, len(t),
                                       x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       v.ctypes.data_as(ctypes.POINTER(ctypes.c_double))), "s1b_orbit_eval_host")
    return x, v


def bounds(poly, start_time, end_time, start_rng, end_rng, hmin, hmax):
    lib = _lib.load()
    out = (ctypes.c_double * 4)()
    _lib.check(lib.s1b_bounds(ctypes.byref(poly), start_time, end_time, start_rng, end_rng, hmin, hmax, out),
               "s1b_bounds")
    return np.array(list(out))


def burst_plan(radar, orbit, fm, dc, burst, rsc=None, allow_empty=True) -> _lib.BurstPlan:
    """One burst's plan (geo2rdr.cu:387-600 host work).  ``orbit`` = (tt, xx, vv);
    ``fm``/``dc`` = [n, 5] tables (time, t0, c0, c1, c2)."""
    lib = _lib.load()
    corb, k1 = c_orbit(*orbit)
    cfm, k2 = c_poly_table(fm)
    cdc, k3 = c_poly_table(dc)
    crad = c_radar(radar)
    cb = c_burst(burst)
    crsc = c_rsc(rsc) if rsc is not None else None
    plan = _lib.BurstPlan()
    st = lib.s1b_burst_plan(ctypes.byref(crad), ctypes.byref(corb), ctypes.byref(cfm), ctypes.byref(cdc),
                            ctypes.byref(cb), ctypes.byref(crsc) if crsc is not None else None,
                            ctypes.byref(plan))
    if st == _lib.S1B_ERR_EMPTY and allow_empty:
        return plan
    _lib.check(st, "s1b_burst_plan")
    return plan


def crossmul_box(h1, h2, rowlook, collook, use_union=False):
    """(box [left, top, right, bottom], header6) or (None, header6) for an empty box."""
    lib = _lib.load()
    a = (ctypes.c_int32 * 6)(*[int(v) for v in h1[:6]])
    b = (ctypes.c_int32 * 6)(*[int(v) for v in h2[:6]])
    box = (ctypes.c_int32 * 4)()
    hdr = (ctypes.c_int32 * 6)()
    st = lib.s1b_crossmul_box(a, b, rowlook, collook, 1 if use_union else 0, box, hdr)
    if st == _lib.S1B_ERR_EMPTY:
        return None, list(hdr)
    _lib.check(st, "s1b_crossmul_box")
    return list(box), list(hdr)


def footprint_boxes(acq):
    """Footprint box (latmin, latmax, lonmin, lonmax) of every burst of an
    acquisition (the burst bounds of geo2rdr.cu:387-400), from the planner."""
    return [tuple(float(v) for v in burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, b, None).latlon_box)
            for b in acq.bursts]


def burst_geometry_device(acqs, rsc=None, device="cuda"):
    """Footprint, DEM window (on ``rsc`` when given) and TOPS centre terms of
    every burst of the acquisitions ``acqs`` in one GPU launch
    (``s1b_burst_geometry``).  Returns one ``_lib.BurstGeometry`` per burst, in
    the order of the acquisitions and their bursts."""
    import torch
    orbits, orbit_of, tables, bursts = [], {}, [], []
    for a in acqs:
        key = id(a.orbit)
        if key not in orbit_of:
            orbit_of[key] = len(orbits)
            orbits.append(orbit_poly(*a.orbit))
        for tab in (a.fm, a.dc):
            tables.append(np.asarray(tab, dtype=np.float64).reshape(-1, 5))
        r = a.radar
        for b in a.bursts:
            bursts.append(_lib.BurstGeometryIn(orbit_of[key], len(tables) - 2, len(tables) - 1,
                                               int(r.lines_per_burst), int(r.samples_per_burst), float(b.azimuth_time),
                                               float(r.prf), float(r.azimuth_time_interval),
                                               float(r.slant_range_time), float(r.range_sampling_rate),
                                               float(r.radar_frequency), float(r.azimuth_steering_rate),
                                               float(r.hmin), float(r.hmax)))
    max_rec = max(len(t) for t in tables)
    packed = np.zeros((len(tables), max_rec, 5), dtype=np.float64)
    for i, t in enumerate(tables):
        packed[i, :len(t)] = t
    counts = np.array([len(t) for t in tables], dtype=np.int32)

    def dev_bytes(obj):
        raw = bytes(obj) if not isinstance(obj, np.ndarray) else obj.tobytes()
        return torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device)

    d_orb = dev_bytes((_lib.OrbitPoly * len(orbits))(*orbits))
    d_tab = dev_bytes(packed)
    d_cnt = dev_bytes(counts)
    d_in = dev_bytes((_lib.BurstGeometryIn * len(bursts))(*bursts))
    out = torch.empty(len(bursts) * ctypes.sizeof(_lib.BurstGeometry), dtype=torch.uint8, device=device)
    crsc = c_rsc(rsc) if rsc is not None else None
    _lib.check(_lib.load().s1b_burst_geometry(_lib.dptr(d_orb), len(orbits), _lib.dptr(d_tab), _lib.dptr(d_cnt),
                                              len(tables), max_rec, _lib.dptr(d_in), len(bursts),
                                              ctypes.byref(crsc) if crsc is not None else None, _lib.dptr(out),
                                              _lib.stream_ptr()), "s1b_burst_geometry")
    raw = bytes(out.cpu().numpy())
    n = ctypes.sizeof(_lib.BurstGeometry)
    return [_lib.BurstGeometry.from_buffer_copy(raw[i * n:(i + 1) * n]) for i in range(len(bursts))]
