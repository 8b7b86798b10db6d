"""Float64 oracle of the radar-grid coregistration chain (no reference
counterpart; the north-star mode of the build).

Test infrastructure only (see ``oracle/__init__.py``).

Given float64 lat/lon/height rasters of the reference radar grid, the
secondary burst is resampled onto that grid:
  1. geo2rdr of every reference pixel on the secondary orbit -> secondary
     (azimuth, range) sample coordinates; stored as offsets relative to the
     reference pixel index (same formulas as the reference geo2rdr,
     csrc/src/geo2rdr.cu:197-207, with the orbit of orbit.cu);
  2. the secondary is deramped (geo2rdr.cu:138-158 formula), interpolated at
     those coordinates (8-tap windowed sinc, or bilinear as geo2rdr.cu:220-237)
     and reramped with its own TOPS phase at the fractional position;
  3. coherence with a 5 x 5 boxcar |sum conj(r) s| / sqrt(sum|r|^2 sum|s|^2).

Interpolation kernel (8 taps, k = -3..4 around n0 = floor(x), f = x - n0):
    w_k = sinc(k - f) * (0.5 + 0.5 cos(pi (k - f) / 4)),  normalised to sum 1.
"""
from __future__ import annotations

import math

import numpy as np

from . import geometry as og
from .geo2rdr import SOL, PI, BurstCoeffs

TAPS = np.arange(-3, 5)


def sinc8_weights(f):
    """[..., 8] normalised windowed-sinc weights at fractional offsets f in [0, 1)."""
    f = np.asarray(f, dtype=np.float64)[..., None]
    x = TAPS - f
    w = np.sinc(x) * (0.5 + 0.5 * np.cos(PI * x / 4.0))
    return w / w.sum(axis=-1, keepdims=True)


def offsets(lat, lon, hgt, radar, orbit, burst_time):
    """Secondary sample coordinates of reference pixels -> (az_off, rg_off, az, rg).

    lat/lon/hgt: float64 [L, S] of the reference grid.  az/rg are the absolute
    secondary sample coordinates; the offsets subtract the reference pixel
    index (row, column)."""
    tt, xx, vv = orbit
    L, S = lat.shape
    llh = np.stack([lat, lon, hgt], axis=-1)
    xyz = og.llh2xyz(llh)
    dtaz = 1.0 / radar.prf
    tend = burst_time + (radar.lines_per_burst - 1) * dtaz
    tmid = 0.5 * (burst_time + tend)
    xm, vm = og.intp_orbit(tt, xx, vv, np.float64(tmid))
    tline, dr, _ = og.orbitrangetime(tt, xx, vv, xyz, tmid, xm, vm)
    rng = np.sqrt((dr * dr).sum(-1))
    rngstart = radar.slant_range_time * SOL / 2.0
    dmrg = SOL / 2.0 / radar.range_sampling_rate
    rg = (rng - rngstart) / dmrg
    az = (tline - burst_time) / dtaz
    rows = np.arange(L, dtype=np.float64)[:, None]
    cols = np.arange(S, dtype=np.float64)[None, :]
    return az - rows, rg - cols, az, rg


def tops_phase(radar, co: BurstCoeffs, az, rg):
    """TOPS phase -pi kt (eta - etaref)^2 at fractional secondary coordinates
    (the deramp formula of geo2rdr.cu:151-152 with kt, etaref evaluated at the
    continuous range sample and eta at the continuous line)."""
    ati = radar.azimuth_time_interval
    L = radar.lines_per_burst
    tr = radar.slant_range_time + rg / radar.range_sampling_rate
    fm0, fm1, fm2, fm3 = co.fm
    dc0, dc1, dc2, dc3 = co.dc
    ka = fm1 + (tr - fm0) * (fm2 + fm3 * (tr - fm0))
    fnc = dc1 + (tr - dc0) * (dc2 + dc3 * (tr - dc0))
    kt = ka * co.ks / (ka - co.ks)
    etaref = -fnc / ka - co.etac0
    eta = -L * ati / 2.0 + az * ati
    d = eta - etaref
    return -PI * kt * d * d


def resample(sec, radar, co: BurstCoeffs, az, rg, interp="sinc8", exact=False):
    """Deramp, interpolate at (az, rg), reramp; zero where the kernel leaves
    the burst.  sec: complex64 [L, S] as acquired (TOPS-modulated).  Returns
    complex64, or complex128 with ``exact``."""
    L, S = sec.shape
    rows = np.arange(L, dtype=np.float64)[:, None]
    cols = np.arange(S, dtype=np.float64)[None, :]
    der = sec.astype(np.complex128) * np.exp(1j * tops_phase(radar, co, rows, cols))
    n_a = np.floor(az).astype(np.int64)
    n_r = np.floor(rg).astype(np.int64)
    fa = az - n_a
    fr = rg - n_r
    out = np.zeros(az.shape, dtype=np.complex128)
    if interp == "sinc8":
        ok = (n_a - 3 >= 0) & (n_a + 4 < L) & (n_r - 3 >= 0) & (n_r + 4 < S)
        wa = sinc8_weights(fa[ok])
        wr = sinc8_weights(fr[ok])
        na, nr = n_a[ok], n_r[ok]
        acc = np.zeros(na.shape, dtype=np.complex128)
        for i, ka in enumerate(TAPS):
            row = np.zeros(na.shape, dtype=np.complex128)
            for j, kr in enumerate(TAPS):
                row += wr[:, j] * der[na + ka, nr + kr]
            acc += wa[:, i] * row
        out[ok] = acc
    else:
        ok = (n_a >= 0) & (n_a + 1 < L) & (n_r >= 0) & (n_r + 1 < S)
        na, nr, a, r = n_a[ok], n_r[ok], fa[ok], fr[ok]
        c1 = der[na, nr] * (1 - r) + der[na, nr + 1] * r
        c2 = der[na + 1, nr] * (1 - r) + der[na + 1, nr + 1] * r
        out[ok] = c1 * (1 - a) + c2 * a
    out *= np.exp(-1j * tops_phase(radar, co, az, rg))
    out[~ok] = 0
    return (out if exact else out.astype(np.complex64)), ok


def box_coherence(ref, sec, win=5):
    """|sum conj(r) s| / sqrt(sum |r|^2 sum |s|^2) over win x win boxes (float64),
    windows clipped at the image border; 0 where the denominator is 0."""
    r = ref.astype(np.complex128)
    s = sec.astype(np.complex128)
    h = win // 2

    def box(a):
        p = np.pad(a, h)
        c = np.cumsum(np.cumsum(p, 0), 1)
        c = np.pad(c, ((1, 0), (1, 0)))
        n0, n1 = a.shape
        return (c[win:win + n0, win:win + n1] - c[:n0, win:win + n1] - c[win:win + n0, :n1] + c[:n0, :n1])

    num = np.abs(box(np.conj(r) * s))
    # the cumulative-sum differences can leave tiny negative residues where a
    # box is all zeros
    den = np.sqrt(np.maximum(box(np.abs(r) ** 2).real, 0) * np.maximum(box(np.abs(s) ** 2).real, 0))
    with np.errstate(invalid="ignore", divide="ignore"):
        g = np.where(den > 0, num / np.where(den > 0, den, 1), 0.0)
    return g
