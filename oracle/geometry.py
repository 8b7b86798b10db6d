"""FP64 geometry oracle: ellipsoid conversions, orbit Hermite interpolation,
zero-Doppler Newton and burst footprint bounds.

Test infrastructure only (see ``oracle/__init__.py``).

Follows, operation for operation where it matters for rounding:
  * ``csrc/include/orbit.hpp:6-11``  WGS84 constants
  * ``csrc/src/orbit.cu:15-35``      llh2xyz
  * ``csrc/src/orbit.cu:37-70``      xyz2llh
  * ``csrc/src/orbit.cu:170-222``    orbithermite (4-point Hermite)
  * ``csrc/src/orbit.cu:224-245``    intp_orbit (truncating window rule)
  * ``csrc/src/orbit.cu:247-280``    orbitrangetime (51 iterations, 5e-9 s)
  * ``csrc/src/bounds.cu:7-317``     bounds / rah2ll / geodesic heading
  * ``s1proc/orbit.py:84-166``       Python interpolant (closest window) and Newton
  * ``s1proc/utils.py:240-292``      _los: LOS vectors and look angles of a grid

All functions are vectorised over leading axes with NumPy float64.
"""
from __future__ import annotations

import math

import numpy as np

RA = 6378137.0  # orbit.hpp:7-8
RE2 = 0.00669437999015  # orbit.hpp:9-11
SOL = 299792458.0  # geo2rdr.cu:26-28
PI = math.pi


def llh2xyz(llh, r_a=RA, r_e2=RE2):
    """Geodetic (deg, deg, m) -> ECEF (m).  orbit.cu:15-35."""
    llh = np.asarray(llh, dtype=np.float64)
    r_lat = llh[..., 0] * PI / 180
    r_lon = llh[..., 1] * PI / 180
    h = llh[..., 2]
    coslat = np.cos(r_lat)
    coslon = np.cos(r_lon)
    sinlat = np.sin(r_lat)
    sinlon = np.sin(r_lon)
    re = r_a / np.sqrt(1.0 - r_e2 * sinlat * sinlat)
    x = (re + h) * coslat * coslon
    y = (re + h) * coslat * sinlon
    z = (re * (1 - r_e2) + h) * sinlat
    return np.stack([x, y, z], axis=-1)


def xyz2llh(xyz, r_a=RA, r_e2=RE2):
    """ECEF (m) -> geodetic (deg, deg, m), one-step Bowring.  orbit.cu:37-70."""
    xyz = np.asarray(xyz, dtype=np.float64)
    x = xyz[..., 0]
    y = xyz[..., 1]
    z = xyz[..., 2]
    r_q2 = 1.0 / (1.0 - r_e2)
    r_q = math.sqrt(r_q2)
    r_q3 = r_q2 - 1.0
    r_b = r_a * math.sqrt(1 - r_e2)
    lon = np.arctan2(y, x)
    lon = np.where((y < 0) & (lon > 0), lon - PI, lon)
    lon = np.where((y > 0) & (lon < 0), lon + PI, lon)
    r_p = np.sqrt(x * x + y * y)
    r_tant = (z / r_p) * r_q
    r_theta = np.arctan(r_tant)
    r_tant = (z + r_q3 * r_b * np.sin(r_theta) ** 3) / (
        r_p - r_e2 * r_a * np.cos(r_theta) ** 3)
    lat = np.arctan(r_tant)
    r_re = r_a / np.sqrt(1.0 - r_e2 * np.sin(lat) * np.sin(lat))
    h = r_p / np.cos(lat) - r_re
    return np.stack([lat / PI * 180, lon / PI * 180, h], axis=-1)


def orbithermite(tt, xx, vv, t):
    """4-point Hermite position/velocity.  orbit.cu:170-222.

    tt: [..., 4]; xx, vv: [..., 4, 3]; t: [...] -> (satx [..., 3], satv [..., 3]).
    The loop order and operation order of the reference are kept so that the
    non-FMA host build of the reference and this function agree to the last bit
    except for libm differences.
    """
    tt = np.asarray(tt, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    shape = t.shape
    li = [np.ones(shape) for _ in range(4)]
    a, b, a2, b2 = [None] * 4, [None] * 4, [None] * 4, [None] * 4
    for i in range(4):
        dl = np.zeros(shape)
        hdot = np.zeros(shape)
        for j in range(4):
            if i == j:
                continue
            dl = dl + 1.0 / (tt[..., i] - tt[..., j])
            li[i] = li[i] * (t - tt[..., j]) / (tt[..., i] - tt[..., j])
            p = 1.0 / (tt[..., i] - tt[..., j])
            for k in range(4):
                if k == i or k == j:
                    continue
                p = p * (t - tt[..., k]) / (tt[..., i] - tt[..., k])
            hdot = hdot + p
        l2 = li[i] * li[i]
        a[i] = (1 - 2 * (t - tt[..., i]) * dl) * l2
        b[i] = (t - tt[..., i]) * l2
        a2[i] = -2 * dl * l2 + (1 - 2 * (t - tt[..., i]) * dl) * li[i] * 2 * hdot
        b2[i] = l2 + (t - tt[..., i]) * li[i] * 2 * hdot
    satx = np.zeros(shape + (3,))
    satv = np.zeros(shape + (3,))
    for j in range(3):
        sx = np.zeros(shape)
        sv = np.zeros(shape)
        for i in range(4):
            sx = sx + (a[i] * xx[..., i, j] + b[i] * vv[..., i, j])
            sv = sv + (a2[i] * xx[..., i, j] + b2[i] * vv[..., i, j])
        satx[..., j] = sx
        satv[..., j] = sv
    return satx, satv


def orbit_window(tt, t):
    """Window start index used by intp_orbit.  orbit.cu:229-232.

    ``int ilocation = (t - t0) / (t1 - t0)`` truncates toward zero, then the
    index is clamped to [1, n-3]; the window is [ilocation-1, ilocation+2].
    """
    tt = np.asarray(tt, dtype=np.float64)
    n = tt.shape[0]
    q = (np.asarray(t, dtype=np.float64) - tt[0]) / (tt[1] - tt[0])
    il = np.trunc(q)
    il = np.where(il > 1, il, 1)
    il = np.where(il < n - 3, il, n - 3)
    return il.astype(np.int64)


def intp_orbit(tt, xx, vv, t):
    """Orbit position/velocity at time t.  orbit.cu:224-245.

    tt [n], xx/vv [n, 3], t [...] -> (satx [..., 3], satv [..., 3]).
    """
    tt = np.asarray(tt, dtype=np.float64)
    xx = np.asarray(xx, dtype=np.float64).reshape(-1, 3)
    vv = np.asarray(vv, dtype=np.float64).reshape(-1, 3)
    il = orbit_window(tt, t)
    idx = il[..., None] - 1 + np.arange(4)
    return orbithermite(tt[idx], xx[idx], vv[idx], t)


def orbitrangetime(tt, xx, vv, xyz, tline0, satx0, satv0, max_iter=51, tol=5.0e-9):
    """Zero-Doppler time by fixed-point Newton.  orbit.cu:247-280.

    Vectorised over the leading axes of ``xyz`` [..., 3].  Each element stops
    iterating (is frozen) once |tline - tprev| < tol, exactly as the reference
    loop breaks.  Returns (tline [...], dr [..., 3], iterations [...]).
    """
    xyz = np.asarray(xyz, dtype=np.float64)
    shape = xyz.shape[:-1]
    tline = np.full(shape, float(tline0))
    satx = np.broadcast_to(np.asarray(satx0, dtype=np.float64), shape + (3,)).copy()
    satv = np.broadcast_to(np.asarray(satv0, dtype=np.float64), shape + (3,)).copy()
    active = np.ones(shape, dtype=bool)
    iters = np.zeros(shape, dtype=np.int64)
    for _ in range(max_iter):
        if not active.any():
            break
        ia = np.nonzero(active.ravel())[0]
        tl = tline.reshape(-1)[ia]
        sx = satx.reshape(-1, 3)[ia]
        sv = satv.reshape(-1, 3)[ia]
        p = xyz.reshape(-1, 3)[ia]
        tprev = tl
        fn = np.zeros(tl.shape)
        fnprime = np.zeros(tl.shape)
        for i in range(3):
            dri = p[:, i] - sx[:, i]
            fn = fn + dri * sv[:, i]
            fnprime = fnprime - sv[:, i] * sv[:, i]
        tl = tl - fn / fnprime
        nx, nv = intp_orbit(tt, xx, vv, tl)
        tline.reshape(-1)[ia] = tl
        satx.reshape(-1, 3)[ia] = nx
        satv.reshape(-1, 3)[ia] = nv
        iters.reshape(-1)[ia] += 1
        done = np.abs(tl - tprev) < tol
        flat_active = active.reshape(-1)
        flat_active[ia[done]] = False
    dr = xyz - satx
    return tline, dr, iters


def interp_orbit_closest(tt, xx, vv, t):
    """The Python orbit interpolant: the 4-point Hermite window around the
    state vector closest to t (argmin |t - tt|, clamped to [1, n-3]).
    s1proc/orbit.py:84-115.  tt [n], xx/vv [n, 3], t [...]."""
    tt = np.asarray(tt, dtype=np.float64)
    xx = np.asarray(xx, dtype=np.float64).reshape(-1, 3)
    vv = np.asarray(vv, dtype=np.float64).reshape(-1, 3)
    t = np.asarray(t, dtype=np.float64)
    il = np.abs(t[..., None] - tt).argmin(axis=-1)
    il = np.minimum(np.maximum(il, 1), tt.shape[0] - 3)
    idx = il[..., None] - 1 + np.arange(4)
    return orbithermite(tt[idx], xx[idx], vv[idx], t)


def orbitrangetime_py(tt, xx, vv, xyz, tline0, satx0, satv0):
    """s1proc/orbit.py:118-166 (the numba loop), vectorised over points: the
    same fixed-point step and 5e-9 s stop on the closest-sample interpolant.
    Returns (dr [..., 3], tline [...])."""
    xyz = np.asarray(xyz, dtype=np.float64)
    shape = xyz.shape[:-1]
    tline = np.full(shape, float(tline0))
    satx = np.broadcast_to(np.asarray(satx0, dtype=np.float64), shape + (3,)).copy()
    satv = np.broadcast_to(np.asarray(satv0, dtype=np.float64), shape + (3,)).copy()
    active = np.ones(shape, dtype=bool)
    for _ in range(51):
        if not active.any():
            break
        ia = np.nonzero(active.ravel())[0]
        tl = tline.reshape(-1)[ia]
        sx = satx.reshape(-1, 3)[ia]
        sv = satv.reshape(-1, 3)[ia]
        dr = xyz.reshape(-1, 3)[ia] - sx
        fn = dr[:, 0] * sv[:, 0] + dr[:, 1] * sv[:, 1] + dr[:, 2] * sv[:, 2]
        fnprime = -sv[:, 0] * sv[:, 0] - sv[:, 1] * sv[:, 1] - sv[:, 2] * sv[:, 2]
        tprev = tl
        tl = tl - fn / fnprime
        nx, nv = interp_orbit_closest(tt, xx, vv, tl)
        tline.reshape(-1)[ia] = tl
        satx.reshape(-1, 3)[ia] = nx
        satv.reshape(-1, 3)[ia] = nv
        active.reshape(-1)[ia[np.abs(tl - tprev) < 5.0e-9]] = False
    return xyz - satx, tline


def los_grid(orb, dem, latmax, lonmin, dlat, dlon, nlat, nlon):
    """LOS unit vectors (float32 [n, 3]) and look angles (float32 [nlat, nlon],
    degrees) of an RSC grid.  s1proc/utils.py:240-292 (_los): the grid of
    geocoordinates.py:114-118 (numpy.mgrid from latmax to latmin, lonmin to
    lonmax, with latmin/lonmax from geocoordinates.py:70-71), llh2xyz_vec and
    orbitrangetime from the middle state vector (orbit.py:168-188), the float32
    cast, then the look angle from the float32 vectors."""
    orb = np.asarray(orb, dtype=np.float64)
    tt, xx, vv = orb[:, 0], orb[:, 1:4], orb[:, 4:7]
    latmin = latmax + dlat * (nlat - 1)
    lonmax = lonmin + dlon * (nlon - 1)
    lat, lon = np.mgrid[latmax:latmin:(nlat * 1j), lonmin:lonmax:(nlon * 1j)]
    llh = np.column_stack((lat.flatten(), lon.flatten(), np.asarray(dem).flatten()))
    xyz = llh2xyz(llh)
    nmid = len(tt) // 2
    dr, _ = orbitrangetime_py(tt, xx, vv, xyz, tt[nmid], xx[nmid], vv[nmid])
    losvec = (dr / np.sqrt(dr[:, 0] * dr[:, 0] + dr[:, 1] * dr[:, 1] + dr[:, 2] * dr[:, 2])[:, None])
    losvec = losvec.astype(np.float32)
    r_lat = np.radians(lat.flatten())
    r_lon = np.radians(lon.flatten())
    r_n = -np.column_stack([np.cos(r_lat) * np.cos(r_lon), np.cos(r_lat) * np.sin(r_lon), np.sin(r_lat)])
    costheta = np.clip(np.sum(losvec * r_n, axis=1).reshape(nlat, nlon), -1, 1)
    theta = np.rad2deg(np.arccos(costheta)).astype(np.float32)
    return losvec, theta


# --------------------------------------------------------------------------
# Burst footprint bounds (host side of geo2rdr).  bounds.cu:7-317.
# Scalar code: 8 corner points per burst.
# --------------------------------------------------------------------------

def _sign(v):
    return float((v > 0) - (v < 0))  # bounds.cu:31


def _reast(r_lat, r_a=RA, r_e2=RE2):  # bounds.cu:33-35
    return r_a / math.sqrt(1.0 - r_e2 * math.pow(math.sin(r_lat), 2))


def _rnorth(r_lat, r_a=RA, r_e2=RE2):  # bounds.cu:37-39
    return r_a * (1.0 - r_e2) / math.pow(1.0 - r_e2 * math.pow(math.sin(r_lat), 2), 1.5)


def _rdir(r_lat, hdg, r_a=RA, r_e2=RE2):  # bounds.cu:41-45
    re = _reast(r_lat, r_a, r_e2)
    rn = _rnorth(r_lat, r_a, r_e2)
    return (re * rn) / (re * math.pow(math.cos(hdg), 2) + rn * math.pow(math.sin(hdg), 2))


def _normalize(v):  # bounds.cu:49-53
    n = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
    return [v[0] / n, v[1] / n, v[2] / n]


def _dot(a, b):  # bounds.cu:55-57
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]


def _cross(a, b):  # bounds.cu:59-64
    return [a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]]


def _tcnbasis(pos, vel, look_dir="RIGHT"):  # bounds.cu:66-92
    llh = xyz2llh(np.asarray(pos))
    r_lat = float(llh[0]) * PI / 180.0
    r_lon = float(llh[1]) * PI / 180.0
    r_n = [-math.cos(r_lat) * math.cos(r_lon), -math.cos(r_lat) * math.sin(r_lon), -math.sin(r_lat)]
    if look_dir == "RIGHT":
        r_temp = _cross(r_n, vel)
    else:
        r_temp = _cross(vel, r_n)
    r_c = _normalize(r_temp)
    r_t = _normalize(_cross(r_c, r_n))
    return r_t, r_c, r_n


def _ellipsoidal_hdg(ll1, ll2, r_a=RA, r_e2=RE2):  # bounds.cu:112-199
    r_e = math.sqrt(r_e2)
    r_sqrtome2 = math.sqrt(1.0 - r_e2)
    r_f = 1.0 - r_sqrtome2
    r_ep = r_e * r_f / (r_e2 - r_f)
    r_n = r_f / r_e2
    r_k1 = (16.0 * r_e2 * r_n * r_n + r_ep * r_ep) / (r_ep * r_ep)
    r_k2 = (16.0 * r_e2 * r_n * r_n) / (16.0 * r_e2 * r_n * r_n + r_ep * r_ep)
    r_k3 = (16.0 * r_e2 * r_n * r_n) / (r_ep * r_ep)
    r_k4 = (16.0 * r_n - r_ep * r_ep) / (16.0 * r_e2 * r_n * r_n + r_ep * r_ep)
    r_k5 = 16.0 / (r_e2 * (16.0 * r_e2 * r_n * r_n + r_ep * r_ep))
    rad = lambda d: d * PI / 180.0  # bounds.cu:27
    r_tanlati = math.tan(rad(ll1[0]))
    r_tanlatf = math.tan(rad(ll2[0]))
    r_l = abs(rad(ll2[1]) - rad(ll1[1]))
    r_lsign = rad(ll2[1]) - rad(ll1[1])
    r_sinlon = math.sin(r_l)
    r_coslon = math.cos(r_l)
    r_tanbetai = r_sqrtome2 * r_tanlati
    r_tanbetaf = r_sqrtome2 * r_tanlatf
    r_cosbetai = 1.0 / math.sqrt(1.0 + r_tanbetai * r_tanbetai)
    r_cosbetaf = 1.0 / math.sqrt(1.0 + r_tanbetaf * r_tanbetaf)
    r_sinbetai = r_tanbetai * r_cosbetai
    r_sinbetaf = r_tanbetaf * r_cosbetaf
    r_ac = r_sinbetai * r_sinbetaf
    r_bc = r_cosbetai * r_cosbetaf
    r_cosphi = r_ac + r_bc * r_coslon
    r_sinphi = _sign(r_sinlon) * math.sqrt(1.0 - min(r_cosphi * r_cosphi, 1.0))
    r_phi = abs(math.atan2(r_sinphi, r_cosphi))
    if r_a * abs(r_phi) > 1e-6:
        r_ca = (r_bc * r_sinlon) / r_sinphi
        r_cb = r_ca * r_ca
        r_cc = (r_cosphi * (1.0 - r_cb)) / r_k1
        r_cd = (-2.0 * r_ac) / r_k1
        r_ce = -r_ac * r_k2
        r_cf = r_k3 * r_cc
        r_cg = r_phi * r_phi / r_sinphi
        r_x = ((r_phi * (r_k4 + r_cb) + r_sinphi * (r_cc + r_cd) + r_cg * (r_cf + r_ce)) * r_ca) / r_k5
        r_lambda = r_l + r_x
        r_sinlam = math.sin(r_lambda)
        r_coslam = math.cos(r_lambda)
        r_t2 = (r_tanbetaf * r_cosbetai - r_coslam * r_sinbetai)
        r_sinlon = r_sinlam * _sign(r_lsign)
        return math.atan2(r_sinlon, r_t2)
    return 0.0


def rah2ll(rah, tt, xx, vv, start_time, end_time, look_dir="RIGHT"):
    """(range, time, height) corners -> lat/lon.  bounds.cu:237-286."""
    xyzs, _ = intp_orbit(tt, xx, vv, np.float64(start_time))
    xyze, _ = intp_orbit(tt, xx, vv, np.float64(end_time))
    xyzm, _ = intp_orbit(tt, xx, vv, np.float64((start_time + end_time) / 2.0))
    llhs = xyz2llh(xyzs)
    llhe = xyz2llh(xyze)
    hdg = _ellipsoidal_hdg([float(llhs[0]), float(llhs[1])], [float(llhe[0]), float(llhe[1])])
    llhm = xyz2llh(xyzm)
    rcurv = _rdir(float(llhm[0]) * PI / 180.0, hdg)
    dopfact = 0.0
    lat = np.zeros(len(rah))
    lon = np.zeros(len(rah))
    for i, (r, t, h) in enumerate(rah):
        xyz, vel = intp_orbit(tt, xx, vv, np.float64(t))
        xyz = [float(c) for c in xyz]
        vel = [float(c) for c in vel]
        llh = xyz2llh(np.asarray(xyz))
        vhat = _normalize(vel)
        that, chat, nhat = _tcnbasis(xyz, vel, look_dir)
        aa = rcurv + float(llh[2])
        bb = rcurv + h
        costheta = 0.5 * ((aa / r + r / aa - bb / aa * bb / r))
        sintheta = math.sqrt(1.0 - costheta * costheta)
        gamm = costheta * r
        alpha = (dopfact * r - gamm * _dot(nhat, vhat)) / _dot(vhat, that)
        beta = math.sqrt((r * sintheta) * (r * sintheta) - alpha * alpha)
        tar = [xyz[j] + (gamm * nhat[j] + alpha * that[j] + beta * chat[j]) for j in range(3)]
        llt = xyz2llh(np.asarray(tar))
        lat[i] = llt[0]
        lon[i] = llt[1]
    return lat, lon


def bounds(start_time, end_time, start_rng, end_rng, hmin, hmax, tt, xx, vv, look_dir="RIGHT"):
    """Burst footprint lat/lon box [latmin, latmax, lonmin, lonmax].  bounds.cu:288-317."""
    rah = []
    for i in range(8):
        r = start_rng if i < 4 else end_rng
        t = start_time if i % 4 < 2 else end_time
        h = hmin if i % 2 == 0 else hmax
        rah.append((r, t, h))
    lat, lon = rah2ll(rah, tt, xx, vv, start_time, end_time, look_dir)
    return np.array([lat.min(), lat.max(), lon.min(), lon.max()])
