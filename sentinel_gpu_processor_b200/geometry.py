"""s1proc's geometry call surface on the GPU, with its names, arguments and
return layouts (s1proc/geometry.py:150-241, s1proc/orbit.py:84-188):
``llh2xyz``, ``xyz2llh`` and their ``_vec`` forms, ``interp_orbit``,
``orbitrangetime``, ``orbitrangetime_vec``, and ``los`` (s1proc/utils.py:240-292,
``_los``: line-of-sight vectors and look angles of a DEM grid).

Arrays are numpy in and out like the numba originals; the arithmetic runs
in libs1b (float64).  The orbit is the reference interpolant as window
polynomials (agreement 5.6e-9 m).  The window follows the CUDA executables'
rule int((t - t0)/dt) (csrc/src/orbit.cu:224-245); the numba interp_orbit
takes the closest state vector instead, which selects the same 4-point
Hermite except within half a state-vector spacing of a window change.  The
zero-Doppler iteration is the exact Newton, stopping at the same 5e-9 s.
"""
from __future__ import annotations

import numpy as np
import torch

from . import kernels, plan as _plan


def _dev():
    return torch.device("cuda", torch.cuda.current_device())


def llh2xyz_vec(llh):
    """[n, 3] (deg, deg, m) -> [n, 3] ECEF (m)."""
    x = torch.as_tensor(np.asarray(llh, dtype=np.float64).reshape(-1, 3), device=_dev())
    return kernels.llh2xyz(x).cpu().numpy()


def llh2xyz(llh):
    """One point (deg, deg, m) -> ECEF [3]."""
    return llh2xyz_vec(np.asarray(llh, dtype=np.float64)[None, :])[0]


def xyz2llh_vec(xyz):
    """[n, 3] ECEF (m) -> [n, 3] (deg, deg, m), one-step Bowring."""
    x = torch.as_tensor(np.asarray(xyz, dtype=np.float64).reshape(-1, 3), device=_dev())
    return kernels.xyz2llh(x).cpu().numpy()


def xyz2llh(xyz):
    return xyz2llh_vec(np.asarray(xyz, dtype=np.float64)[None, :])[0]


def interp_orbit(timeorbit, xx, vv, t):
    """Position and velocity at time t (scalar -> [3], [3]; array -> [n, 3], [n, 3])."""
    poly = _plan.orbit_poly(np.asarray(timeorbit), np.asarray(xx), np.asarray(vv))
    x, v = _plan.orbit_eval(poly, t)
    if np.ndim(t) == 0:
        return x[0], v[0]
    return x, v


def orbitrangetime(timeorbit, xx, vv, xyz, tline0, satx0=None, satv0=None):
    """Zero-Doppler (dr, tline) of one point (or of [n, 3] points): dr = xyz - X(tline).
    ``satx0``/``satv0`` are accepted for the reference signature; the Newton
    starts from ``tline0`` on the orbit itself."""
    poly = _plan.orbit_poly(np.asarray(timeorbit), np.asarray(xx), np.asarray(vv))
    p = np.asarray(xyz, dtype=np.float64)
    one = p.ndim == 1
    t, dr = kernels.zero_doppler(poly, torch.as_tensor(p.reshape(-1, 3), device=_dev()), float(tline0))
    t, dr = t.cpu().numpy(), dr.cpu().numpy()
    return (dr[0], float(t[0])) if one else (dr, t)


def orbitrangetime_vec(llh, tt, xx, vv):
    """Unit line-of-sight vectors [n, 3] of points [n, 3] (deg, deg, m),
    each solved from the middle state vector (s1proc/orbit.py:167-188)."""
    tt = np.asarray(tt, dtype=np.float64)
    poly = _plan.orbit_poly(tt, np.asarray(xx), np.asarray(vv))
    xyz = kernels.llh2xyz(torch.as_tensor(np.asarray(llh, dtype=np.float64).reshape(-1, 3), device=_dev()))
    _, dr = kernels.zero_doppler(poly, xyz, float(tt[len(tt) // 2]))
    return (dr / dr.norm(dim=1, keepdim=True)).cpu().numpy()


def los(orb, dem, rsc):
    """LOS unit vectors and look angles of every pixel of an RSC grid, as
    s1proc/utils.py:240-292 (``_los``) computes them, in one kernel.

    ``orb``: [n, 7] rows (time, x, y, z, vx, vy, vz); ``dem``: int16 heights,
    nlat * nlon values; ``rsc``: an object with latmax, lonmin, dlat, dlon,
    nlat, nlon (``formats.read_rsc`` or the reference's GeoCoordinates).
    Returns (losvec float32 [nlat * nlon, 3], theta float32 [nlat, nlon]
    degrees).  The grid is numpy.mgrid's (geocoordinates.py:70-71, 114-118);
    each point's zero-Doppler time is solved from the middle state vector's
    time (orbit.py:168-188)."""
    orb = np.asarray(orb, dtype=np.float64)
    tt, xx, vv = orb[:, 0], orb[:, 1:4], orb[:, 4:7]
    poly = _plan.orbit_poly(tt, xx, vv)
    nlat, nlon = int(rsc.nlat), int(rsc.nlon)
    latmin = rsc.latmax + rsc.dlat * (nlat - 1)
    lonmax = rsc.lonmin + rsc.dlon * (nlon - 1)
    # numpy.mgrid with a complex step: start + index * ((stop - start) / (num - 1))
    lat_step = (latmin - rsc.latmax) / float(nlat - 1) if nlat > 1 else 0.0
    lon_step = (lonmax - rsc.lonmin) / float(nlon - 1) if nlon > 1 else 0.0
    d = torch.as_tensor(np.ascontiguousarray(np.asarray(dem, dtype=np.int16).reshape(nlat, nlon)), device=_dev())
    losvec, theta = kernels.los_grid(poly, tt[len(tt) // 2], rsc.latmax, lat_step, rsc.lonmin, lon_step, d)
    return losvec.cpu().numpy(), theta.cpu().numpy()
