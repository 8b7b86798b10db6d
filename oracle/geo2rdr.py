"""FP64 oracle of the reference ``geo2rdr`` executable (one burst at a time).

Test infrastructure only (see ``oracle/__init__.py``).

Follows ``csrc/src/geo2rdr.cu``:
  * 48-59    closest_sample
  * 86-128   find_first_last_nonzero_rows_kernel, 273-299 host wrapper
  * 138-158  deramp_burst
  * 170-248  reproject (per DEM pixel: llh2xyz, orbitrangetime, validity
             window, per-pixel kt/etaref, bilinear, reramp + range phase)
  * 387-400  per-burst bounds, 408-422 DEM window sizing
  * 469-542  host deramp coefficients (ks, FM/DC interpolation, kt, etaref)
  * 569-600  DEM window, tstart/tmid/xmid/vmid
  * 620-650  non-zero-row crop and ``.gslc`` header
The interpolation of the reference runs in double precision with float
operands (``float * double`` promotes); this oracle does the same in float64
and rounds the stored results to complex64 as the reference does.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import geometry as geo

SOL = 299792458.0
PI = math.pi


@dataclass
class Radar:
    """The per-subswath DB keys read at geo2rdr.cu:333-376."""
    samples_per_burst: int
    lines_per_burst: int
    prf: float
    wvl: float
    hmin: float
    hmax: float
    range_sampling_rate: float
    slant_range_time: float
    azimuth_steering_rate: float
    azimuth_time_interval: float
    radar_frequency: float


@dataclass
class BurstMeta:
    """Per-burst DB keys (geo2rdr.cu:365-376)."""
    azimuth_time: float
    first_valid_line: int
    last_valid_line: int
    first_valid_sample: int
    last_valid_sample: int


def closest_sample(t, t0):
    """geo2rdr.cu:48-59 (first index of the minimum |t - t0|)."""
    idx = 0
    mindist = 1e10
    for i, ti in enumerate(t):
        dist = abs(ti - t0)
        if mindist > dist:
            mindist = dist
            idx = i
    return idx


def interp_poly(table, tc):
    """Linear interpolation of (t0, c0, c1, c2) at time tc.  geo2rdr.cu:485-527.

    table: array [n, 5] with columns (time, t0, c0, c1, c2).
    Returns (t0, c0, c1, c2) -- note the reference interpolates c0,c1,c2 first
    and t0 last; the values are independent so the order is irrelevant.
    """
    time = table[:, 0]
    n = len(time)
    idx = closest_sample(time, tc)
    cols = table[:, 1:5]
    if time[idx] < tc and idx < n - 1:
        frac = (tc - time[idx]) / (time[idx + 1] - time[idx])
        out = cols[idx] + frac * (cols[idx + 1] - cols[idx])
    elif time[idx] > tc and idx > 0:
        frac = (tc - time[idx - 1]) / (time[idx] - time[idx - 1])
        out = cols[idx - 1] + frac * (cols[idx] - cols[idx - 1])
    else:
        out = cols[idx].copy()
    return tuple(float(v) for v in out)  # t0, c0, c1, c2


@dataclass
class BurstCoeffs:
    ks: float
    fm: tuple  # (t0, c0, c1, c2)
    dc: tuple
    kt: np.ndarray  # [S]
    etaref: np.ndarray  # [S]
    etac0: float
    eta: np.ndarray  # [L]


def burst_coefficients(radar: Radar, orbit, fmtab, dctab, burst: BurstMeta) -> BurstCoeffs:
    """Host deramp coefficients.  geo2rdr.cu:469-542."""
    tt, xx, vv = orbit
    L = radar.lines_per_burst
    S = radar.samples_per_burst
    ati = radar.azimuth_time_interval
    tc = burst.azimuth_time + L * ati / 2  # 477-478
    _, vpoint = geo.intp_orbit(tt, xx, vv, np.float64(tc))
    vpoint = [float(v) for v in vpoint]
    vs = math.sqrt(vpoint[0] * vpoint[0] + vpoint[1] * vpoint[1] + vpoint[2] * vpoint[2])
    ks = 2.0 * vs * radar.radar_frequency / SOL * radar.azimuth_steering_rate * PI / 180.0
    fm = interp_poly(fmtab, tc)
    dc = interp_poly(dctab, tc)
    i = np.arange(L, dtype=np.float64)
    eta = -L * ati / 2.0 + i * ati  # 529-532
    col = np.arange(S, dtype=np.float64)
    trange = radar.slant_range_time + col / radar.range_sampling_rate  # 534
    dt = trange - fm[0]
    ka = fm[1] + dt * (fm[2] + fm[3] * dt)
    dt = trange - dc[0]
    fnc = dc[1] + dt * (dc[2] + dc[3] * dt)
    kt = ka * ks / (ka - ks)
    etac = -fnc / ka
    etaref = etac - etac[0]
    return BurstCoeffs(ks=ks, fm=fm, dc=dc, kt=kt, etaref=etaref, etac0=float(etac[0]), eta=eta)


def deramp(burst: np.ndarray, co: BurstCoeffs) -> np.ndarray:
    """deramp_burst, geo2rdr.cu:138-158: burst * exp(-i*pi*kt*(eta-etaref)^2).

    The product is formed in float64 from the complex64 input and rounded to
    complex64, like the reference's ``Complex = double * double`` stores.
    """
    etadiff = co.eta[:, None] - co.etaref[None, :]
    phase = -PI * co.kt[None, :] * etadiff * etadiff
    bx = np.cos(phase)
    by = np.sin(phase)
    ax = burst.real.astype(np.float64)
    ay = burst.imag.astype(np.float64)
    out = np.empty(burst.shape, dtype=np.complex64)
    out.real = (ax * bx - ay * by).astype(np.float32)
    out.imag = (ax * by + ay * bx).astype(np.float32)
    return out


@dataclass
class Rsc:
    nlat: int
    nlon: int
    latmax: float
    lonmin: float
    dlat: float
    dlon: float


@dataclass
class GeoWindow:
    left: int
    top: int
    right: int
    bottom: int

    @property
    def nrow(self):
        return self.bottom - self.top

    @property
    def ncol(self):
        return self.right - self.left


def burst_latlon_box(radar: Radar, orbit, burst: BurstMeta):
    """geo2rdr.cu:387-400 -> [latmin, latmax, lonmin, lonmax]."""
    tt, xx, vv = orbit
    tstart = burst.azimuth_time
    dtaz = 1.0 / radar.prf
    tend = tstart + (radar.lines_per_burst - 1) * dtaz
    rngstart = radar.slant_range_time * SOL / 2.0
    dmrg = SOL / 2.0 / radar.range_sampling_rate
    rngend = rngstart + (radar.samples_per_burst - 1) * dmrg
    return geo.bounds(tstart, tend, rngstart, rngend, radar.hmin, radar.hmax, tt, xx, vv, "RIGHT")


def dem_window(latlon, rsc: Rsc):
    """geo2rdr.cu:569-586 (C ``int()`` truncation, then clamping)."""
    latmin, latmax, lonmin, lonmax = [float(v) for v in latlon]
    left = int((lonmin - rsc.lonmin) / rsc.dlon)
    top = int((latmax - rsc.latmax) / rsc.dlat)
    right = int((lonmax - rsc.lonmin) / rsc.dlon + 1)
    bottom = int((latmin - rsc.latmax) / rsc.dlat + 1)
    left = max(0, left)
    top = max(0, top)
    right = min(rsc.nlon, right)
    bottom = min(rsc.nlat, bottom)
    return GeoWindow(left, top, right, bottom)


def reproject(dem_win: np.ndarray, deramped: np.ndarray, radar: Radar, orbit, burst: BurstMeta,
              co: BurstCoeffs, latmax0: float, lonmin0: float, dlat: float, dlon: float,
              return_offsets: bool = False):
    """reproject kernel, geo2rdr.cu:170-248, for a whole DEM window.

    dem_win: int16 [nrow, ncol]; deramped: complex64 [L, S].
    Returns complex64 [nrow, ncol] (and the float64 (azoff, rgoff, valid) maps
    when ``return_offsets``).
    """
    tt, xx, vv = orbit
    nrow, ncol = dem_win.shape
    L = radar.lines_per_burst
    S = radar.samples_per_burst
    tstart = burst.azimuth_time
    dtaz = 1.0 / radar.prf
    tend = tstart + (L - 1) * dtaz
    tmid = (tstart + tend) * 0.5
    rngstart = radar.slant_range_time * SOL / 2.0
    dmrg = SOL / 2.0 / radar.range_sampling_rate
    xmid, vmid = geo.intp_orbit(tt, xx, vv, np.float64(tmid))
    row = np.arange(nrow, dtype=np.float64)[:, None]
    col = np.arange(ncol, dtype=np.float64)[None, :]
    lat = np.broadcast_to(latmax0 + row * dlat, (nrow, ncol))
    lon = np.broadcast_to(lonmin0 + col * dlon, (nrow, ncol))
    h = dem_win.astype(np.float64)
    xyz = geo.llh2xyz(np.stack([lat, lon, h], axis=-1))
    tline, dr, _ = geo.orbitrangetime(tt, xx, vv, xyz, tmid, xmid, vmid)
    rngpix = np.sqrt(dr[..., 0] * dr[..., 0] + dr[..., 1] * dr[..., 1] + dr[..., 2] * dr[..., 2])
    rgoff = (rngpix - rngstart) / dmrg
    azoff = (tline - tstart) / dtaz
    valid = ((rgoff > burst.first_valid_sample) & (rgoff < burst.last_valid_sample - 1)
             & (azoff >= burst.first_valid_line + 5) & (azoff < burst.last_valid_line - 5))
    out = np.zeros((nrow, ncol), dtype=np.complex64)
    if valid.any():
        R = rngpix[valid]
        t = tline[valid]
        fmt0, fmc0, fmc1, fmc2 = co.fm
        dct0, dcc0, dcc1, dcc2 = co.dc
        dt = R * 2 / SOL - fmt0
        ka = fmc0 + dt * (fmc1 + fmc2 * dt)
        dt = R * 2 / SOL - dct0
        fnc = dcc0 + dt * (dcc1 + dcc2 * dt)
        kt = ka * co.ks / (ka - co.ks)
        etac = -fnc / ka
        etaref = etac - co.etac0
        eta = -L * dtaz / 2.0 + t - tstart
        etadiff = eta - etaref
        reramp = -PI * kt * etadiff * etadiff
        ro = rgoff[valid]
        ao = azoff[valid]
        intr = np.trunc(ro).astype(np.int64)
        fracr = ro - intr
        inta = np.trunc(ao).astype(np.int64)
        fraca = ao - inta
        flat = deramped.reshape(-1)
        i1 = inta * S + intr
        b1, b2 = flat[i1], flat[i1 + 1]
        b3, b4 = flat[i1 + S], flat[i1 + S + 1]

        def lerp(u, v, f):  # float * double in double, stored to float
            re = (u.real.astype(np.float64) * (1 - f) + v.real.astype(np.float64) * f).astype(np.float32)
            im = (u.imag.astype(np.float64) * (1 - f) + v.imag.astype(np.float64) * f).astype(np.float32)
            return re, im

        c1r, c1i = lerp(b1, b2, fracr)
        c2r, c2i = lerp(b3, b4, fracr)
        resx = c1r.astype(np.float64) * (1 - fraca) + c2r.astype(np.float64) * fraca
        resy = c1i.astype(np.float64) * (1 - fraca) + c2i.astype(np.float64) * fraca
        phase = 4.0 * PI / radar.wvl * R - reramp
        cp = np.cos(phase)
        sp = np.sin(phase)
        vals = np.empty(R.shape, dtype=np.complex64)
        vals.real = (resx * cp - resy * sp).astype(np.float32)
        vals.imag = (resx * sp + resy * cp).astype(np.float32)
        out[valid] = vals
    if return_offsets:
        return out, azoff, rgoff, valid
    return out


def window_offsets(dem_win: np.ndarray, rows, radar: Radar, orbit, burst: BurstMeta, latmax0: float,
                   lonmin0: float, dlat: float, dlon: float):
    """(azoff, rgoff) float64 [len(rows), ncol] of the given rows of a DEM
    window, as reproject forms them (geo2rdr.cu:195-207: llh2xyz at
    lat = latmax0 + row dlat, lon = lonmin0 + col dlon, orbitrangetime seeded
    at the burst centre, then the line and sample of tline and |dr|)."""
    tt, xx, vv = orbit
    rows = np.asarray(rows, dtype=np.int64)
    ncol = dem_win.shape[1]
    L = radar.lines_per_burst
    tstart = burst.azimuth_time
    dtaz = 1.0 / radar.prf
    tmid = (tstart + (tstart + (L - 1) * dtaz)) * 0.5
    rngstart = radar.slant_range_time * SOL / 2.0
    dmrg = SOL / 2.0 / radar.range_sampling_rate
    xmid, vmid = geo.intp_orbit(tt, xx, vv, np.float64(tmid))
    lat = np.broadcast_to((latmax0 + rows.astype(np.float64) * dlat)[:, None], (len(rows), ncol))
    lon = np.broadcast_to((lonmin0 + np.arange(ncol, dtype=np.float64) * dlon)[None, :], (len(rows), ncol))
    h = dem_win[rows].astype(np.float64)
    xyz = geo.llh2xyz(np.stack([lat, lon, h], axis=-1))
    tline, dr, _ = geo.orbitrangetime(tt, xx, vv, xyz, tmid, xmid, vmid)
    rngpix = np.sqrt(dr[..., 0] * dr[..., 0] + dr[..., 1] * dr[..., 1] + dr[..., 2] * dr[..., 2])
    return (tline - tstart) / dtaz, (rngpix - rngstart) / dmrg


def nonzero_rows(out: np.ndarray):
    """find_nonzero_rows, geo2rdr.cu:86-128 + 273-299: (first, last_excl) or None."""
    nz = np.any((out.real != 0) | (out.imag != 0), axis=1)
    if not nz.any():
        return None
    idx = np.nonzero(nz)[0]
    return int(idx[0]), int(idx[-1]) + 1


def geo2rdr_burst(slc: np.ndarray, dem: np.ndarray, rsc: Rsc, radar: Radar, orbit, fmtab, dctab,
                  burst: BurstMeta):
    """One burst of geo2rdr.cu:466-651.

    slc: complex64 [L, S] (TOPS-modulated, as read from the input);
    dem: int16 [rsc.nlat, rsc.nlon].
    Returns (header int32[64], data complex64 [rows, ncol]) or None when the
    reference would skip the burst (empty window or no non-zero rows).
    """
    co = burst_coefficients(radar, orbit, fmtab, dctab, burst)
    der = deramp(slc, co)
    box = burst_latlon_box(radar, orbit, burst)
    w = dem_window(box, rsc)
    if w.left >= w.right or w.top >= w.bottom:
        return None
    dem_win = dem[w.top:w.bottom, w.left:w.right]
    out = reproject(dem_win, der, radar, orbit, burst, co,
                    rsc.latmax + rsc.dlat * w.top, rsc.lonmin + rsc.dlon * w.left,
                    rsc.dlat, rsc.dlon)
    nz = nonzero_rows(out)
    if nz is None or nz[0] == nz[1]:
        return None
    first, last = nz
    header = np.zeros(64, dtype=np.int32)
    header[0] = rsc.nlat
    header[1] = rsc.nlon
    header[2] = w.left
    header[3] = w.top + first
    header[4] = w.right
    header[5] = w.top + last
    return header, out[first:last].copy()
