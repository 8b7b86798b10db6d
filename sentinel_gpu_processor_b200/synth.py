"""Seeded synthetic Sentinel-1 IW scenes.

The reference benchmarks on real Sentinel-1 data that cannot be used here;
these generators stand in for it with the shapes, geometry and value
distributions of the workload: a C-band radar (lambda = 0.05546576 m, range
spacing 2.329562 m, azimuth interval 2.055556e-3 s, near range 8.0e5 m), a
circular orbit at 693 km and 7.6 km/s sampled by 11 state vectors 10 s
apart, a secondary orbit offset by a perpendicular baseline, fractal (fBm,
H = 0.8) terrain on a 1/7200-degree lat/lon grid, circular-Gaussian speckle
and TOPS azimuth modulation with a chosen Doppler rate.

Everything here is host-side input preparation.  Tensors are made with torch
(CPU or CUDA) so that large scenes are generated on the device.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import formats

SOL = 299792458.0
RA = 6378137.0
RE2 = 0.00669437999015

WAVELENGTH = 0.05546576
RANGE_SPACING = 2.329562
AZIMUTH_INTERVAL = 2.055556e-3
NEAR_RANGE = 8.0e5
ALTITUDE = 693.0e3
SPEED = 7600.0
INCLINATION_DEG = 98.18
ORBIT_T0 = 50000.0
ORBIT_DT = 10.0
ORBIT_N = 11
GEO_STEP = 1.0 / 7200.0


@dataclass
class Radar:
    """Per-subswath radar parameters (the keys geo2rdr reads, geo2rdr.cu:333-376)."""
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
class Burst:
    azimuth_time: float
    first_valid_line: int
    last_valid_line: int
    first_valid_sample: int
    last_valid_sample: int


@dataclass
class Acquisition:
    """One SLC (one date) of one subswath: radar, orbit, FM/DC tables, bursts."""
    radar: Radar
    orbit: tuple  # (tt [n], xx [n,3], vv [n,3]) float64
    fm: np.ndarray  # [n, 5] (time, t0, c0, c1, c2)
    dc: np.ndarray
    bursts: list


@dataclass
class PairScene:
    """A reference/secondary pair of bursts over one DEM grid."""
    name: str
    seed: int
    ref: list  # list[Acquisition], one per burst group (per burst for uneven sizes)
    sec: list
    rsc: formats.Rsc
    dem: object  # torch int16 [nlat, nlon]
    ref_slc: list  # list of torch complex64 [L, S] per burst (TOPS-modulated)
    sec_slc: list
    rowlook: int
    collook: int
    alpha: float
    n_win: int = 32
    extra: dict = field(default_factory=dict)

    @property
    def burst_pixels(self):
        return sum(int(s.shape[0]) * int(s.shape[1]) for s in self.ref_slc)


# ----------------------------------------------------------------------------
# Small geodesy helpers (numpy) for scene layout
# ----------------------------------------------------------------------------

def _llh2xyz(lat, lon, h):
    lat = np.radians(lat)
    lon = np.radians(lon)
    re = RA / np.sqrt(1.0 - RE2 * np.sin(lat) ** 2)
    return np.stack([(re + h) * np.cos(lat) * np.cos(lon), (re + h) * np.cos(lat) * np.sin(lon),
                     (re * (1 - RE2) + h) * np.sin(lat)], axis=-1)


def _xyz2llh(xyz):
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    lon = np.arctan2(y, x)
    p = np.hypot(x, y)
    lat = np.arctan2(z, p * (1 - RE2))
    for _ in range(6):
        n = RA / np.sqrt(1 - RE2 * np.sin(lat) ** 2)
        h = p / np.cos(lat) - n
        lat = np.arctan2(z, p * (1 - RE2 * n / (n + h)))
    n = RA / np.sqrt(1 - RE2 * np.sin(lat) ** 2)
    h = p / np.cos(lat) - n
    return np.degrees(lat), np.degrees(lon), h


def make_orbit(lat_c=35.0, lon_c=10.0, t_c=ORBIT_T0 + 50.0, altitude=ALTITUDE, speed=SPEED,
               n=ORBIT_N, dt=ORBIT_DT, t0=ORBIT_T0, inclination=INCLINATION_DEG, offset=(0.0, 0.0, 0.0)):
    """Circular ECEF orbit through the sub-satellite point (lat_c, lon_c) at t_c, ascending."""
    r = RA + altitude
    inc = math.radians(inclination)
    u_c = math.asin(math.sin(math.radians(lat_c)) / math.sin(inc))
    # longitude of the node such that the sub-satellite longitude at u_c is lon_c
    dl = math.atan2(math.cos(inc) * math.sin(u_c), math.cos(u_c))
    om = math.radians(lon_c) - dl
    e1 = np.array([math.cos(om), math.sin(om), 0.0])
    e2 = np.array([-math.cos(inc) * math.sin(om), math.cos(inc) * math.cos(om), math.sin(inc)])
    w = speed / r
    tt = t0 + dt * np.arange(n, dtype=np.float64)
    u = u_c + w * (tt - t_c)
    xx = r * (np.cos(u)[:, None] * e1 + np.sin(u)[:, None] * e2) + np.asarray(offset)[None, :]
    vv = r * w * (-np.sin(u)[:, None] * e1 + np.cos(u)[:, None] * e2)
    return tt, xx, vv


def _orbit_at(orbit, t):
    tt, xx, vv = orbit
    # the orbit is a circle: interpolate the angle exactly from two samples
    k = int(np.clip(np.searchsorted(tt, t) - 1, 0, len(tt) - 2))
    a = (t - tt[k]) / (tt[k + 1] - tt[k])
    p0, p1 = xx[k], xx[k + 1]
    v0 = vv[k]
    r = np.linalg.norm(p0)
    ang = math.acos(np.clip(np.dot(p0, p1) / (r * np.linalg.norm(p1)), -1, 1))
    e1 = p0 / r
    e2 = v0 / np.linalg.norm(v0)
    th = a * ang
    p = r * (math.cos(th) * e1 + math.sin(th) * e2)
    v = np.linalg.norm(v0) * (-math.sin(th) * e1 + math.cos(th) * e2)
    return p, v


def rdr2geo(orbit, t, rng, h):
    """Ground point (lat, lon) at zero Doppler, slant range ``rng``, height ``h``, right-looking."""
    p, v = _orbit_at(orbit, t)
    lat, lon, _ = _xyz2llh(p)
    n_hat = -np.array([math.cos(math.radians(lat)) * math.cos(math.radians(lon)),
                       math.cos(math.radians(lat)) * math.sin(math.radians(lon)),
                       math.sin(math.radians(lat))])
    c_hat = np.cross(n_hat, v)
    c_hat /= np.linalg.norm(c_hat)
    n2 = np.cross(v, c_hat)
    n2 /= np.linalg.norm(n2)  # down direction orthogonal to v
    lo, hi = 0.0, math.radians(85.0)
    for _ in range(80):
        th = 0.5 * (lo + hi)
        g = p + rng * (math.cos(th) * n2 + math.sin(th) * c_hat)
        _, _, hg = _xyz2llh(g)
        if hg > h:  # the look ray rises with the angle: too far out
            hi = th
        else:
            lo = th
    g = p + rng * (math.cos(th) * n2 + math.sin(th) * c_hat)
    la, lo_, _ = _xyz2llh(g)
    return float(la), float(lo_), th


# ----------------------------------------------------------------------------
# Radar, TOPS tables, bursts
# ----------------------------------------------------------------------------

def make_radar(lines, samples, near_range=NEAR_RANGE, steering_rate=1.590368784, hmin=-100.0, hmax=3100.0):
    ati = AZIMUTH_INTERVAL
    return Radar(samples_per_burst=int(samples), lines_per_burst=int(lines), prf=1.0 / ati,
                 wvl=WAVELENGTH, hmin=float(hmin), hmax=float(hmax),
                 range_sampling_rate=SOL / (2.0 * RANGE_SPACING),
                 slant_range_time=2.0 * near_range / SOL, azimuth_steering_rate=float(steering_rate),
                 azimuth_time_interval=ati, radar_frequency=SOL / WAVELENGTH)


def tops_tables(radar: Radar, t_c: float, kt_target: float, vs: float = SPEED):
    """FM-rate and Doppler-centroid tables whose kt at near range, burst centre, is ``kt_target``.

    ks = 2 vs f0 / c * steering_rate * pi / 180 (geo2rdr.cu:482-483) and the
    reference forms kt = ka ks / (ka - ks) (geo2rdr.cu:539), so the FM rate
    is ka = kt ks / (kt - ks).  Three table entries around the burst centre
    with small coefficient changes exercise the time interpolation.
    """
    ks = 2.0 * vs * radar.radar_frequency / SOL * radar.azimuth_steering_rate * math.pi / 180.0
    ka = kt_target * ks / (kt_target - ks)
    swath_t = radar.samples_per_burst / radar.range_sampling_rate
    t0 = radar.slant_range_time
    fm, dc = [], []
    for k, dtk in enumerate((-2.75, 0.25, 3.25)):
        s = 1.0 + 0.002 * (k - 1)
        fm.append([t_c + dtk, t0, ka * s, 0.02 * ka / swath_t, 0.0])
        dc.append([t_c + dtk, t0, 30.0 * s, -4.0e4, 1.0e6])
    return np.asarray(fm), np.asarray(dc)


def burst_meta(t_start, lines, samples, margin_l=24, margin_s=40):
    return Burst(azimuth_time=float(t_start), first_valid_line=margin_l, last_valid_line=lines - margin_l,
                 first_valid_sample=margin_s, last_valid_sample=samples - margin_s)


def tops_coefficients(acq: Acquisition, burst: Burst):
    """kt[S], etaref[S], eta[L] of a burst (the host formulas of geo2rdr.cu:469-542)."""
    r = acq.radar
    L, S = r.lines_per_burst, r.samples_per_burst
    tc = burst.azimuth_time + L * r.azimuth_time_interval / 2
    vs = SPEED
    ks = 2.0 * vs * r.radar_frequency / SOL * r.azimuth_steering_rate * math.pi / 180.0

    def interp(tab):
        i = int(np.argmin(np.abs(tab[:, 0] - tc)))
        if tab[i, 0] < tc and i < len(tab) - 1:
            f = (tc - tab[i, 0]) / (tab[i + 1, 0] - tab[i, 0])
            return tab[i, 1:] + f * (tab[i + 1, 1:] - tab[i, 1:])
        if tab[i, 0] > tc and i > 0:
            f = (tc - tab[i - 1, 0]) / (tab[i, 0] - tab[i - 1, 0])
            return tab[i - 1, 1:] + f * (tab[i, 1:] - tab[i - 1, 1:])
        return tab[i, 1:].copy()

    fm = interp(acq.fm)
    dc = interp(acq.dc)
    tr = r.slant_range_time + np.arange(S) / r.range_sampling_rate
    ka = fm[1] + (tr - fm[0]) * (fm[2] + fm[3] * (tr - fm[0]))
    fnc = dc[1] + (tr - dc[0]) * (dc[2] + dc[3] * (tr - dc[0]))
    kt = ka * ks / (ka - ks)
    etac = -fnc / ka
    etaref = etac - etac[0]
    eta = -L * r.azimuth_time_interval / 2.0 + np.arange(L) * r.azimuth_time_interval
    return kt, etaref, eta


# ----------------------------------------------------------------------------
# Terrain and speckle (torch)
# ----------------------------------------------------------------------------

def _hash01(ix, iy, octave, seed, torch):
    """Uniform [0,1) lattice values from a 32-bit integer hash (Wang/Jenkins style mixing)."""
    h = (ix * 374761393 + iy * 668265263 + octave * 2147483647 + seed * 1274126177) & 0xFFFFFFFF
    h = ((h ^ (h >> 13)) * 1274126177) & 0xFFFFFFFF
    h = (h ^ (h >> 16)) & 0xFFFFFFFF
    return h.to(torch.float32) * (1.0 / 4294967296.0)


def fbm_height(lat, lon, seed, hmax, H=0.8, base_deg=0.2, octaves=9):
    """Fractal terrain in [0, hmax] m evaluated at (lat, lon) degrees (torch float64 tensors).

    Sum of value-noise octaves with amplitude 2^(-k H) (fBm with Hurst
    exponent H); lattice values come from a hash of the global lattice index,
    so any window of the globe is generated consistently.
    """
    import torch
    acc = torch.zeros_like(lat, dtype=torch.float32)
    norm = 0.0
    for k in range(octaves):
        cell = base_deg / (2 ** k)
        u = lat / cell
        v = lon / cell
        iu = torch.floor(u)
        iv = torch.floor(v)
        fu = (u - iu).to(torch.float32)
        fv = (v - iv).to(torch.float32)
        fu = fu * fu * (3 - 2 * fu)
        fv = fv * fv * (3 - 2 * fv)
        iu = iu.to(torch.int64)
        iv = iv.to(torch.int64)
        v00 = _hash01(iu, iv, k, seed, torch)
        v10 = _hash01(iu + 1, iv, k, seed, torch)
        v01 = _hash01(iu, iv + 1, k, seed, torch)
        v11 = _hash01(iu + 1, iv + 1, k, seed, torch)
        n = (v00 * (1 - fu) * (1 - fv) + v10 * fu * (1 - fv) + v01 * (1 - fu) * fv + v11 * fu * fv)
        a = 2.0 ** (-k * H)
        acc += a * (n - 0.5)
        norm += a
    z = acc / norm
    z = (z - z.min()) / max(float(z.max() - z.min()), 1e-6)
    return z * hmax


def make_dem(rsc: formats.Rsc, seed, hmax, device="cpu"):
    import torch
    lat = rsc.latmax + rsc.dlat * torch.arange(rsc.nlat, dtype=torch.float64, device=device)[:, None]
    lon = rsc.lonmin + rsc.dlon * torch.arange(rsc.nlon, dtype=torch.float64, device=device)[None, :]
    lat, lon = torch.broadcast_tensors(lat, lon)
    h = fbm_height(lat, lon, seed, hmax)
    return torch.round(h).to(torch.int16).contiguous()


def speckle(lines, samples, gen, device):
    import torch
    z = torch.randn((lines, samples, 2), generator=gen, device=device, dtype=torch.float32)
    z *= math.sqrt(0.5)
    return torch.view_as_complex(z)


def band_limited_speckle(lines, samples, gen, device, band=0.8):
    """Unit-power circular-Gaussian speckle whose spectrum is flat over the
    central ``band`` of the sampling rate in both axes and zero outside (a
    Sentinel-1 SLC is oversampled by about 1.2 in range and azimuth).  Values
    between samples are then fixed by the samples, so two grids that sample
    one scene at shifted positions see correlated values."""
    import torch
    z = torch.fft.fft2(speckle(lines, samples, gen, device))
    ka = torch.fft.fftfreq(lines, device=device).abs() <= band / 2
    kr = torch.fft.fftfreq(samples, device=device).abs() <= band / 2
    z *= ka[:, None].to(z.dtype)
    z *= kr[None, :].to(z.dtype)
    z = torch.fft.ifft2(z)
    z /= math.sqrt(float(ka.sum()) * float(kr.sum()) / (lines * samples))
    return z.to(torch.complex64)


def tops_modulate(slc, acq: Acquisition, burst: Burst, sign=+1.0):
    """Multiply by exp(sign * i pi kt (eta - etaref)^2) (inverse of the deramp)."""
    import torch
    kt, etaref, eta = tops_coefficients(acq, burst)
    dev = slc.device
    kt = torch.as_tensor(kt, dtype=torch.float64, device=dev)
    etaref = torch.as_tensor(etaref, dtype=torch.float64, device=dev)
    eta = torch.as_tensor(eta, dtype=torch.float64, device=dev)
    d = eta[:, None] - etaref[None, :]
    ph = sign * math.pi * kt[None, :] * d * d
    ph = torch.remainder(ph, 2 * math.pi).to(torch.float32)
    return slc * torch.polar(torch.ones_like(ph), ph)


# ----------------------------------------------------------------------------
# Scenes
# ----------------------------------------------------------------------------

CONFIGS = {
    # name: (lines, samples, rowlook, collook, alpha, hmax, kt)
    "tiny": (96, 320, 2, 4, 0.5, 800.0, -1500.0),
    "small": (160, 640, 2, 8, 0.5, 1500.0, -1500.0),
    "c0": (512, 2048, 2, 8, 0.5, 1500.0, -1500.0),
    "c1": (1500, 21000, 4, 20, 0.6, 3000.0, -1500.0),
}


def _look_angle(r_sat, rng):
    re = RA
    return math.acos((r_sat ** 2 + rng ** 2 - re ** 2) / (2 * r_sat * rng))


def secondary_offset(orbit, t_c, near_range, baseline):
    """ECEF offset of ``baseline`` metres perpendicular to the velocity and to the mid-swath look vector."""
    p, v = _orbit_at(orbit, t_c)
    n_hat = -p / np.linalg.norm(p)
    c_hat = np.cross(n_hat, v)
    c_hat /= np.linalg.norm(c_hat)
    th = _look_angle(np.linalg.norm(p), near_range)
    b_hat = -math.sin(th) * n_hat + math.cos(th) * c_hat
    return baseline * b_hat


def footprint_rsc(acqs, hmin, hmax, margin=0.08, step=GEO_STEP):
    """RSC grid (1/7200 degree) covering every burst footprint, with a margin."""
    lats, lons = [], []
    for acq in acqs:
        r = acq.radar
        for b in acq.bursts:
            t0 = b.azimuth_time
            t1 = t0 + (r.lines_per_burst - 1) * r.azimuth_time_interval
            r0 = r.slant_range_time * SOL / 2
            r1 = r0 + (r.samples_per_burst - 1) * SOL / 2 / r.range_sampling_rate
            for t in (t0, t1):
                for rg in (r0, r1):
                    for h in (hmin, hmax):
                        la, lo, _ = rdr2geo(acq.orbit, t, rg, h)
                        lats.append(la)
                        lons.append(lo)
    la0, la1 = min(lats), max(lats)
    lo0, lo1 = min(lons), max(lons)
    dla = (la1 - la0) * margin
    dlo = (lo1 - lo0) * margin
    latmax = la1 + dla
    lonmin = lo0 - dlo
    nlat = int(math.ceil((la1 - la0 + 2 * dla) / step)) + 1
    nlon = int(math.ceil((lo1 - lo0 + 2 * dlo) / step)) + 1
    return formats.rsc_roundtrip(formats.Rsc(nlat=nlat, nlon=nlon, latmax=latmax, lonmin=lonmin,
                                             dlat=-step, dlon=step))


def make_pair(config="c0", seed=20261203, device="cpu", baseline=150.0, coherence=0.7,
              lines=None, samples=None, rowlook=None, collook=None, alpha=None):
    """A one-burst reference/secondary pair (configs 'tiny', 'small', 'c0', 'c1')."""
    import torch
    L, S, rl, cl, al, hmax, kt = CONFIGS[config]
    L = int(lines or L)
    S = int(samples or S)
    rl = int(rowlook or rl)
    cl = int(collook or cl)
    al = float(alpha if alpha is not None else al)
    rng = np.random.Generator(np.random.PCG64(seed))
    t_c = ORBIT_T0 + 50.0 + float(rng.uniform(-1.0, 1.0))
    orbit_ref = make_orbit(t_c=ORBIT_T0 + 50.0)
    off = secondary_offset(orbit_ref, t_c, NEAR_RANGE + S * RANGE_SPACING / 2, baseline)
    orbit_sec = make_orbit(t_c=ORBIT_T0 + 50.0, offset=off)
    hmin_db, hmax_db = -100.0, hmax + 100.0
    radar = make_radar(L, S, hmin=hmin_db, hmax=hmax_db)
    t_start = t_c - L * AZIMUTH_INTERVAL / 2
    fm, dc = tops_tables(radar, t_c, kt)
    burst = burst_meta(t_start, L, S)
    ref = Acquisition(radar=radar, orbit=orbit_ref, fm=fm, dc=dc, bursts=[burst])
    sec = Acquisition(radar=radar, orbit=orbit_sec, fm=fm.copy(), dc=dc.copy(), bursts=[burst])
    rsc = footprint_rsc([ref, sec], 0.0, hmax)
    dem = make_dem(rsc, seed, hmax, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    s_ref = speckle(L, S, gen, device)
    noise = speckle(L, S, gen, device)
    s_sec = coherence * s_ref + math.sqrt(1 - coherence ** 2) * noise
    ref_slc = tops_modulate(s_ref, ref, burst).contiguous()
    sec_slc = tops_modulate(s_sec, sec, burst).contiguous()
    return PairScene(name=config, seed=seed, ref=[ref], sec=[sec], rsc=rsc, dem=dem,
                     ref_slc=[ref_slc], sec_slc=[sec_slc], rowlook=rl, collook=cl, alpha=al,
                     extra={"hmax": hmax})


def make_frame(seed=20261203, device="cpu", n_swaths=3, n_bursts=9, baseline=150.0,
               line_range=(1480, 1530), sample_range=(20000, 25500), overlap=100,
               kt_range=(-1700.0, -1400.0), coh_range=(0.3, 0.9), rowlook=4, collook=20,
               alpha=0.5, hmax=3000.0, scale=1.0, slc_pairs=None, with_dem=True):
    """A full IW frame: ``n_swaths`` x ``n_bursts`` bursts of uneven size.

    Each burst is its own Acquisition (the reference handles one burst size
    per subswath run).  ``scale`` shrinks line/sample counts for tests.
    ``slc_pairs``: make the SLCs of the first ``slc_pairs`` burst pairs only
    (the others are None); they are the same values as in the whole frame,
    since the speckle of the pairs is drawn in order from one generator.
    ``with_dem=False`` leaves the DEM out (geometry only).
    """
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    orbit_ref = make_orbit(t_c=ORBIT_T0 + 50.0)
    near = [NEAR_RANGE, NEAR_RANGE + 4.6e4, NEAR_RANGE + 9.2e4]
    steer = [1.590368784, 0.979863325, 1.397440818]
    refs, secs, ref_slc, sec_slc, cohs = [], [], [], [], []
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    acq_dur = 0.0
    for sw in range(n_swaths):
        kt = float(rng.uniform(*kt_range))
        off = secondary_offset(orbit_ref, ORBIT_T0 + 50.0, near[sw] + 2.6e4, baseline)
        orbit_sec = make_orbit(t_c=ORBIT_T0 + 50.0, offset=off)
        t = ORBIT_T0 + 50.0 - 0.5 * n_bursts * 2.75
        for b in range(n_bursts):
            L = int(round(rng.integers(line_range[0], line_range[1] + 1) * scale))
            S = int(round(rng.integers(sample_range[0], sample_range[1] + 1) * scale))
            L = max(L, 64)
            S = max(S, 128)
            radar = make_radar(L, S, near_range=near[sw], steering_rate=steer[sw], hmin=-100.0, hmax=hmax + 100.0)
            t_c = t + L * AZIMUTH_INTERVAL / 2
            fm, dc = tops_tables(radar, t_c, kt)
            burst = burst_meta(t, L, S)
            ref = Acquisition(radar=radar, orbit=orbit_ref, fm=fm, dc=dc, bursts=[burst])
            sec = Acquisition(radar=radar, orbit=orbit_sec, fm=fm.copy(), dc=dc.copy(), bursts=[burst])
            g = float(rng.uniform(*coh_range))
            if slc_pairs is None or len(refs) < slc_pairs:
                s_ref = speckle(L, S, gen, device)
                noise = speckle(L, S, gen, device)
                s_sec = g * s_ref + math.sqrt(1 - g * g) * noise
                ref_slc.append(tops_modulate(s_ref, ref, burst).contiguous())
                sec_slc.append(tops_modulate(s_sec, sec, burst).contiguous())
                del s_ref, noise, s_sec
            else:
                ref_slc.append(None)
                sec_slc.append(None)
            refs.append(ref)
            secs.append(sec)
            cohs.append(g)
            t += (L - int(overlap * scale)) * AZIMUTH_INTERVAL
            acq_dur = max(acq_dur, t)
    rsc = footprint_rsc(refs + secs, 0.0, hmax, margin=0.02)
    dem = make_dem(rsc, seed, hmax, device=device) if with_dem else None
    return PairScene(name="frame", seed=seed, ref=refs, sec=secs, rsc=rsc, dem=dem, ref_slc=ref_slc,
                     sec_slc=sec_slc, rowlook=rowlook, collook=collook, alpha=alpha,
                     extra={"coherence": cohs, "hmax": hmax})


def _window(box, rsc):
    """DEM window [left, top, right, bottom) of a footprint box (latmin,
    latmax, lonmin, lonmax) on an RSC grid: C int() truncation of each end
    (csrc/src/geo2rdr.cu:569-586), unclamped."""
    latmin, latmax, lonmin, lonmax = box
    return (int((lonmin - rsc.lonmin) / rsc.dlon), int((latmax - rsc.latmax) / rsc.dlat),
            int((lonmax - rsc.lonmin) / rsc.dlon + 1), int((latmin - rsc.latmax) / rsc.dlat + 1))


def reference_geo2rdr_fits(boxes, rsc):
    """True when the reference geo2rdr's buffers hold every burst window of
    one run.  ``boxes``: the footprint boxes of the bursts of one geo2rdr run.

    geo2rdr.cu:408-423 sizes its host DEM buffer and device output as
    ``int((latmin - latmax)/dlat + 1) x int((lonmax - lonmin)/dlon + 1)`` (max
    over the bursts) while each burst window (569-586) truncates its two ends
    separately and can be one row or column larger; both buffers are flat, so
    the element count must fit."""
    nrow_buf = max(int((b[0] - b[1]) / rsc.dlat + 1) for b in boxes)
    ncol_buf = max(int((b[3] - b[2]) / rsc.dlon + 1) for b in boxes)
    for b in boxes:
        l, t, r, bt = _window(b, rsc)
        l, t, r, bt = max(0, l), max(0, t), min(rsc.nlon, r), min(rsc.nlat, bt)
        if (bt - t) * (r - l) > nrow_buf * ncol_buf:
            return False
    return True


def _axis_terms(b, origin, step, lat):
    """The three C int() arguments of one axis of a burst's footprint: the
    buffer extent (geo2rdr.cu:408-423) and the window's two ends (569-586)."""
    if lat:
        return (b[0] - b[1]) / step + 1, (b[1] - origin) / step, (b[0] - origin) / step + 1
    return (b[3] - b[2]) / step + 1, (b[2] - origin) / step, (b[3] - origin) / step + 1


def reference_safe_rsc(rsc, runs, steps=4000, margin=1e-6):
    """An RSC grid on which the reference geo2rdr stays inside its buffers
    for every run in ``runs`` (a list of footprint-box lists, one per geo2rdr
    run): ``rsc`` itself when it already is, else ``rsc`` with its origin
    moved by a fraction of a pixel (and, when no origin serves every run, its
    spacing stretched by parts per million).  Along each axis the window
    exceeds the buffer exactly when the fractional parts of the window start
    and of the footprint extent add up to one or more, so each axis offset is
    searched on its own.

    A grid is only taken when every int() argument of the windows and
    buffers lies at least ``margin`` pixels from an integer, so the choice is
    the same for footprint boxes that differ in the last bits (the library's
    planner evaluates the orbit through its polynomials, a restatement of
    the reference through the Hermite form).  The values go through the RSC
    text form, as the reference reads them."""
    import math

    def robust(x):
        f = x - math.floor(x)
        return margin < f < 1.0 - margin

    def axis_ok(origin, step, lat):
        for bb in runs:
            terms = [_axis_terms(b, origin, step, lat) for b in bb]
            if not all(robust(x) for t in terms for x in t):
                return False
            buf = max(int(t[0]) for t in terms)
            if max(int(t[2]) - int(t[1]) for t in terms) > buf:
                return False
        return True

    def search(origin0, step, lat, sign):
        for k in range(steps):
            v = float("{0:.14f}".format(origin0 + sign * (k / steps) * abs(step)))
            if axis_ok(v, step, lat):
                return v
        return None

    for m in range(400):
        f = float("{0:.14f}".format(1.0 + 1e-5 * m))
        dlat = float("{0:.14f}".format(rsc.dlat * f)) if m else rsc.dlat
        dlon = float("{0:.14f}".format(rsc.dlon * f)) if m else rsc.dlon
        lat = search(rsc.latmax, dlat, True, +1)
        lon = search(rsc.lonmin, dlon, False, -1)
        if lat is not None and lon is not None:
            out = formats.rsc_roundtrip(formats.Rsc(rsc.nlat, rsc.nlon, lat, lon, dlat, dlon))
            if out == rsc or all(reference_geo2rdr_fits(bb, out) for bb in runs):
                return out
    raise RuntimeError("no DEM grid keeps the reference geo2rdr buffers in bounds")


def regrid(sc: PairScene, rsc) -> PairScene:
    """``sc`` on another RSC grid: the DEM regenerated there (the terrain is
    the same function of latitude and longitude)."""
    import dataclasses
    if rsc == sc.rsc:
        return sc
    dev = sc.dem.device if sc.dem is not None else "cpu"
    return dataclasses.replace(sc, rsc=rsc, dem=make_dem(rsc, sc.seed, sc.extra["hmax"], device=dev))


def on_reference_safe_grid(sc: PairScene, boxes_of, pairs=(0,)) -> PairScene:
    """``sc`` on a DEM grid where the reference geo2rdr, run on each burst of
    the given pairs, stays inside its buffers (``reference_safe_rsc``);
    ``boxes_of(acq)`` gives an acquisition's footprint boxes (the library's
    planner, ``plan.footprint_boxes``, or any restatement of the reference's
    bounds that agrees with it bit for bit)."""
    runs = [boxes_of(a) for k in pairs for a in (sc.ref[k], sc.sec[k])]
    return regrid(sc, reference_safe_rsc(sc.rsc, runs))


@dataclass
class StackScene:
    """A time series of one subswath: a reference date and ``n_sec``
    secondary dates over one DEM grid.  ``ref``: the reference's bursts
    (one Acquisition each); ``sec[d]``: those of secondary date d.  SLCs are
    made on demand (``stack_slc``), so a stack larger than the device's
    memory can be processed in batches of dates."""
    seed: int
    ref: list
    sec: list            # [n_sec][n_bursts] Acquisition
    rsc: formats.Rsc
    dem: object
    days: list           # days after the reference, per secondary date
    baselines: list      # perpendicular baselines (m), per secondary date
    coherence: list      # 0.9 exp(-dt / 60 d), per secondary date
    rowlook: int
    collook: int
    alpha: float
    lines: int
    samples: int
    defo_rate: float = 0.01  # m / yr at the far range edge of the ramp
    extra: dict = field(default_factory=dict)

    @property
    def n_bursts(self):
        return len(self.ref)


def make_stack(seed=20261203 + 5000, device="cpu", n_sec=29, n_bursts=9, lines=1500, samples=21000, overlap=100,
               kt=-1500.0, revisit_days=12, baseline_range=200.0, rowlook=4, collook=20, alpha=0.5, hmax=3000.0,
               with_dem=True):
    """Time-series stack of one subswath: ``n_sec`` secondary dates every
    ``revisit_days`` days after the reference, each with a seeded
    perpendicular baseline uniform in +-``baseline_range`` m and temporal
    coherence 0.9 exp(-dt / 60 d); deformation: a phase ramp across range
    growing at 1 cm/yr (``stack_slc``).  Bursts of ``lines`` x ``samples``,
    consecutive bursts overlapping by ``overlap`` lines."""
    rng = np.random.Generator(np.random.PCG64(seed))
    orbit_ref = make_orbit(t_c=ORBIT_T0 + 50.0)
    near = NEAR_RANGE
    t0 = ORBIT_T0 + 50.0 - 0.5 * n_bursts * 2.75
    radar = make_radar(lines, samples, near_range=near, hmin=-100.0, hmax=hmax + 100.0)
    bursts, t = [], t0
    for _ in range(n_bursts):
        bursts.append((t, burst_meta(t, lines, samples)))
        t += (lines - overlap) * AZIMUTH_INTERVAL
    fm, dc = tops_tables(radar, ORBIT_T0 + 50.0, kt)

    def acqs(orbit):
        return [Acquisition(radar=radar, orbit=orbit, fm=fm.copy(), dc=dc.copy(), bursts=[b]) for _, b in bursts]

    ref = acqs(orbit_ref)
    sec, days, bls, cohs = [], [], [], []
    for d in range(n_sec):
        bl = float(rng.uniform(-baseline_range, baseline_range))
        off = secondary_offset(orbit_ref, ORBIT_T0 + 50.0, near + samples * RANGE_SPACING / 2, bl)
        sec.append(acqs(make_orbit(t_c=ORBIT_T0 + 50.0, offset=off)))
        days.append(revisit_days * (d + 1))
        bls.append(bl)
        cohs.append(0.9 * math.exp(-revisit_days * (d + 1) / 60.0))
    rsc = footprint_rsc(ref + [a for s in sec for a in s], 0.0, hmax, margin=0.02)
    dem = make_dem(rsc, seed, hmax, device=device) if with_dem else None
    return StackScene(seed=seed, ref=ref, sec=sec, rsc=rsc, dem=dem, days=days, baselines=bls, coherence=cohs,
                      rowlook=rowlook, collook=collook, alpha=alpha, lines=lines, samples=samples,
                      extra={"hmax": hmax})


def _stack_cache(st: StackScene, name: str) -> dict:
    return st.extra.setdefault(name, {})


def stack_reference_field(st: StackScene, burst: int, device):
    """The scene of reference burst ``burst`` on its own sample grid, before
    the TOPS modulation: band-limited speckle seeded per burst (cached)."""
    import torch
    cache = _stack_cache(st, "_field")
    if burst not in cache:
        gen = torch.Generator(device=device)
        gen.manual_seed(st.seed * 1000 + burst)
        cache[burst] = band_limited_speckle(st.lines, st.samples, gen, device)
    return cache[burst]


def dem_height_fn(rsc: formats.Rsc, dem):
    """The terrain of a DEM raster as a function of (lat, lon) in degrees:
    bilinear interpolation of its heights (float64), clamped at its edges."""
    import torch
    h = dem.to(torch.float64)
    n0, n1 = h.shape

    def fn(lat, lon):
        y = ((lat - rsc.latmax) / rsc.dlat).clamp(0.0, n0 - 1.0)
        x = ((lon - rsc.lonmin) / rsc.dlon).clamp(0.0, n1 - 1.0)
        y0 = y.floor().clamp(max=n0 - 2).long()
        x0 = x.floor().clamp(max=n1 - 2).long()
        fy, fx = y - y0, x - x0
        a, b = h[y0, x0], h[y0, x0 + 1]
        c, d = h[y0 + 1, x0], h[y0 + 1, x0 + 1]
        return (a + fx * (b - a)) + fy * ((c + fx * (d - c)) - (a + fx * (b - a)))
    return fn


def stack_reference_geometry(st: StackScene, burst: int, device):
    """float64 lat/lon/height rasters of reference burst ``burst``'s samples
    on the stack's DEM, interpolated bilinearly (``rdr2geo_grid``; cached)."""
    cache = _stack_cache(st, "_geom")
    if burst not in cache:
        acq = st.ref[burst]
        cache[burst] = rdr2geo_grid(acq.orbit, acq.radar, acq.bursts[0], dem_height_fn(st.rsc, st.dem.to(device)),
                                    device=device, terrain=True)
    return cache[burst]


def locked_to_reference(field, ref: Acquisition, sec: Acquisition, lat, lon, hgt):
    """``field``, given on the reference burst's sample grid, as the secondary
    acquisition ``sec`` sees it: the value at secondary sample q is the field
    at the reference position p of the same ground point, p + off(p) = q,
    where off is the secondary's geo2rdr of the reference grid (``lat``,
    ``lon``, ``hgt``).  p is found by fixed-point iteration on the bilinearly
    sampled offsets and the field read there by the 8-tap sinc (the s1b
    resampler with the TOPS steering set to zero, i.e. no deramp); its phase
    moves by the change of the point's two-way path between the orbits, so
    that the geocoding, which adds 4 pi R / wvl at each burst's own range,
    brings both back to one value.  Needs CUDA tensors."""
    import dataclasses

    import torch
    import torch.nn.functional as F

    from . import kernels, plan as _plan
    pl = _plan.burst_plan(sec.radar, sec.orbit, sec.fm, sec.dc, sec.bursts[0], None)
    az, rg = kernels.geo2rdr_offsets(pl, lat, lon, hgt)
    L, S = az.shape
    dev = az.device
    qa = torch.arange(L, device=dev, dtype=torch.float32)[:, None]
    qr = torch.arange(S, device=dev, dtype=torch.float32)[None, :]
    off = torch.stack([rg, az])[None]  # grid_sample's x is the range axis
    da, dr = -az, -rg                   # p - q
    for _ in range(3):
        g = torch.stack([(qr + dr) * (2.0 / (S - 1)) - 1.0, (qa + da) * (2.0 / (L - 1)) - 1.0], -1)[None]
        o = F.grid_sample(off, g, mode="bilinear", padding_mode="border", align_corners=True)[0]
        dr, da = -o[0], -o[1]
        del g, o
    flat = dataclasses.replace(ref.radar, azimuth_steering_rate=0.0)
    pl0 = _plan.burst_plan(flat, ref.orbit, ref.fm, ref.dc, ref.bursts[0], None)
    out = kernels.resample(pl0, field.contiguous(), da.contiguous(), dr.contiguous())
    # each ground point's two-way path changes by R_sec - R_ref = dR (q_s - p_s):
    # its phase by -4 pi dR (q_s - p_s) / wvl = 4 pi dR dr / wvl
    k = 4.0 * math.pi * (SOL / 2.0 / sec.radar.range_sampling_rate) / sec.radar.wvl
    ph = torch.remainder(k * dr.double(), 2 * math.pi)
    return out * torch.polar(torch.ones_like(ph), ph).to(torch.complex64)


def ground_lock_pairs(sc: PairScene, pairs) -> PairScene:
    """Make the SLCs of the listed burst pairs of ``sc`` one scene seen by
    both dates, as ``stack_slc`` does for a stack: pair k's reference holds
    band-limited speckle seeded per pair, its ground points come from
    ``rdr2geo_grid(terrain=True)`` on the scene's own DEM, the secondary sees
    the same ground points at its own sample positions
    (``locked_to_reference``) mixed with its own speckle at the pair's
    coherence ``sc.extra["coherence"][k]``; both are TOPS-modulated.  The
    geocoded interferogram of the pair is then coherent at about that
    coherence.  Replaces ``sc.ref_slc[k]`` and ``sc.sec_slc[k]`` in place;
    needs the DEM on a CUDA device."""
    import torch
    dev = sc.dem.device
    height = dem_height_fn(sc.rsc, sc.dem)
    for k in pairs:
        ref, sec = sc.ref[k], sc.sec[k]
        L, S = ref.radar.lines_per_burst, ref.radar.samples_per_burst
        gen = torch.Generator(device=dev)
        gen.manual_seed(sc.seed * 1000 + 7 + k)
        f = band_limited_speckle(L, S, gen, dev)
        lat, lon, hgt = rdr2geo_grid(ref.orbit, ref.radar, ref.bursts[0], height, device=dev, terrain=True)
        s = locked_to_reference(f, ref, sec, lat, lon, hgt)
        del lat, lon, hgt
        g = sc.extra["coherence"][k]
        s = g * s + math.sqrt(1 - g * g) * band_limited_speckle(L, S, gen, dev)
        sc.ref_slc[k] = tops_modulate(f, ref, ref.bursts[0]).contiguous()
        sc.sec_slc[k] = tops_modulate(s, sec, sec.bursts[0]).contiguous()
        del f, s
    return sc


def stack_slc(st: StackScene, date: int, burst: int, device="cpu"):
    """SLC of burst ``burst`` of date ``date`` (-1: the reference), TOPS-
    modulated.  The reference is band-limited speckle seeded per burst on its
    own grid; date d sees that scene from its own orbit: the same ground
    points at its own sample positions (``locked_to_reference``), mixed with
    its own band-limited speckle at the date's coherence, plus the
    deformation phase 4 pi / wvl * rate * dt, the rate a ramp from 0 at near
    range to 1 cm/yr at far range.  Geocoded pairs are then coherent at the
    date's coherence (less the interpolation's own loss).  Secondary dates
    need CUDA (they use the s1b geo2rdr and resampler)."""
    import torch
    L, S = st.lines, st.samples
    f = stack_reference_field(st, burst, device)
    if date < 0:
        return tops_modulate(f, st.ref[burst], st.ref[burst].bursts[0]).contiguous()
    acq = st.sec[date][burst]
    lat, lon, hgt = stack_reference_geometry(st, burst, device)
    s = locked_to_reference(f, st.ref[burst], acq, lat, lon, hgt)
    gen = torch.Generator(device=device)
    gen.manual_seed(st.seed * 1000 + 100000 * (date + 1) + burst)
    g = st.coherence[date]
    s = g * s + math.sqrt(1 - g * g) * band_limited_speckle(L, S, gen, device)
    ramp = torch.linspace(0.0, 1.0, S, dtype=torch.float64, device=device)
    phase = (4 * math.pi / WAVELENGTH * st.defo_rate * st.days[date] / 365.25) * ramp
    s = s * torch.polar(torch.ones_like(phase), phase).to(torch.complex64)[None, :]
    return tops_modulate(s, acq, acq.bursts[0]).contiguous()


def cint16(slc, scale: float = 2000.0):
    """Complex int16 samples (int16 [..., 2], re and im) of a synthetic SLC
    tensor, as a Sentinel-1 measurement TIFF holds them: ``round(scale *
    slc)``, clipped to the int16 range."""
    import torch
    q = torch.stack([slc.real, slc.imag], -1).mul(scale).round().clamp(-32768, 32767)
    return q.to(torch.int16).contiguous()


def frame_pair(frame: PairScene, k: int, margin: int = 64) -> PairScene:
    """Burst pair ``k`` of a frame as its own PairScene, on the part of the
    frame's DEM grid that covers both bursts' footprints (plus a margin)."""
    from . import plan as _plan
    ref, sec = frame.ref[k], frame.sec[k]
    wins = []
    for a in (ref, sec):
        p = _plan.burst_plan(a.radar, a.orbit, a.fm, a.dc, a.bursts[0], frame.rsc)
        wins.append(p.window)
    r = frame.rsc
    left = max(0, min(w[0] for w in wins) - margin)
    top = max(0, min(w[1] for w in wins) - margin)
    right = min(r.nlon, max(w[2] for w in wins) + margin)
    bottom = min(r.nlat, max(w[3] for w in wins) + margin)
    sub = formats.rsc_roundtrip(formats.Rsc(nlat=bottom - top, nlon=right - left, latmax=r.latmax + r.dlat * top,
                                            lonmin=r.lonmin + r.dlon * left, dlat=r.dlat, dlon=r.dlon))
    dem = make_dem(sub, frame.seed, frame.extra["hmax"], device=frame.dem.device)
    return PairScene(name=f"frame[{k}]", seed=frame.seed, ref=[ref], sec=[sec], rsc=sub, dem=dem,
                     ref_slc=[frame.ref_slc[k]], sec_slc=[frame.sec_slc[k]], rowlook=frame.rowlook,
                     collook=frame.collook, alpha=frame.alpha, extra={"hmax": frame.extra["hmax"]})


# ----------------------------------------------------------------------------
# Radar-grid scenes (float64 lat/lon/height rasters of the reference grid)
# ----------------------------------------------------------------------------

def _xyz2llh_t(x, y, z):
    """ECEF -> geodetic by fixed-point iteration (torch float64)."""
    import torch
    lon = torch.atan2(y, x)
    p = torch.sqrt(x * x + y * y)
    lat = torch.atan2(z, p * (1 - RE2))
    for _ in range(5):
        n = RA / torch.sqrt(1 - RE2 * torch.sin(lat) ** 2)
        h = p / torch.cos(lat) - n
        lat = torch.atan2(z, p * (1 - RE2 * n / (n + h)))
    n = RA / torch.sqrt(1 - RE2 * torch.sin(lat) ** 2)
    h = p / torch.cos(lat) - n
    return torch.rad2deg(lat), torch.rad2deg(lon), h


def rdr2geo_grid(orbit, radar, burst, height_fn, device="cpu", outer=4, steps=44, terrain=False):
    """Ground point of every pixel of a burst: zero-Doppler plane at the line
    time, slant range of the sample, on the terrain ``height_fn(lat, lon)``.

    Bisection on the look angle in the plane orthogonal to the velocity
    (right-looking).  ``terrain=True``: for the point where the look ray
    meets the terrain (the ray's height minus the terrain's there changes
    sign; under layover, one of the crossings).  Otherwise ``outer`` rounds
    of: the ray point at the height of the terrain found under the previous
    round's point; on rough terrain these rounds need not reach the surface,
    but the rasters are still points of the pixels' own look rays (the
    radar-grid scenes use them as given).
    Returns float64 (lat, lon, hgt) tensors [lines, samples]."""
    import torch

    from . import plan as _plan
    L, S = radar.lines_per_burst, radar.samples_per_burst
    dtaz = 1.0 / radar.prf
    t = burst.azimuth_time + dtaz * np.arange(L)
    poly = _plan.orbit_poly(*orbit)
    P, V = _plan.orbit_eval(poly, t)
    P = torch.as_tensor(P, dtype=torch.float64, device=device)
    V = torch.as_tensor(V, dtype=torch.float64, device=device)
    d = -P / torch.linalg.norm(P, dim=1, keepdim=True)
    d = d - (d * V).sum(1, keepdim=True) * V / (V * V).sum(1, keepdim=True)
    d = d / torch.linalg.norm(d, dim=1, keepdim=True)
    c = torch.cross(d, V, dim=1)
    c = c / torch.linalg.norm(c, dim=1, keepdim=True)
    r0 = radar.slant_range_time * SOL / 2.0
    R = (r0 + (SOL / 2.0 / radar.range_sampling_rate) * torch.arange(S, dtype=torch.float64, device=device))[None, :]

    def ray_point(th):
        ct, st = torch.cos(th), torch.sin(th)
        gx = P[:, 0:1] + R * (ct * d[:, 0:1] + st * c[:, 0:1])
        gy = P[:, 1:2] + R * (ct * d[:, 1:2] + st * c[:, 1:2])
        gz = P[:, 2:3] + R * (ct * d[:, 2:3] + st * c[:, 2:3])
        return _xyz2llh_t(gx, gy, gz)

    def bisect(below):  # the look angle where below(lat, lon, h) turns false
        lo = torch.zeros((L, S), dtype=torch.float64, device=device)
        hi = torch.full((L, S), math.radians(80.0), dtype=torch.float64, device=device)
        for _ in range(steps):
            th = 0.5 * (lo + hi)
            up = ~below(*ray_point(th))
            hi = torch.where(up, th, hi)
            lo = torch.where(up, lo, th)
        return 0.5 * (lo + hi)

    if terrain:
        return tuple(x.contiguous() for x in
                     ray_point(bisect(lambda la, lo_, hg: hg <= height_fn(la, lo_).to(torch.float64))))
    h = torch.zeros((L, S), dtype=torch.float64, device=device)
    for _ in range(outer):
        lat, lon, hg = ray_point(bisect(lambda la, lo_, hg_: hg_ <= h))
        h = height_fn(lat, lon).to(torch.float64)
    return lat.contiguous(), lon.contiguous(), hg.contiguous()


def reflectivity(lat, lon, seed, lat0, lon0, n_waves=64, min_wavelength=60.0):
    """Band-limited complex random field on the ground (torch complex64):
    a sum of ``n_waves`` plane waves with random directions, wavelengths above
    ``min_wavelength`` metres and random phases, normalised to unit power.
    Both acquisitions sample it at their own ground points, so their images
    of one scene are consistent up to resampling."""
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    north = (lat - lat0) * (math.pi / 180.0 * RA)
    east = (lon - lon0) * (math.pi / 180.0 * RA * math.cos(math.radians(lat0)))
    kmax = 2 * math.pi / min_wavelength
    ang = rng.uniform(0, 2 * math.pi, n_waves)
    kmag = kmax * np.sqrt(rng.uniform(0.0, 1.0, n_waves))
    ph = rng.uniform(0, 2 * math.pi, n_waves)
    amp = rng.standard_normal(n_waves) + 1j * rng.standard_normal(n_waves)
    acc = torch.zeros(lat.shape, dtype=torch.complex128, device=lat.device)
    for k in range(n_waves):
        arg = kmag[k] * (math.cos(ang[k]) * north + math.sin(ang[k]) * east) + ph[k]
        acc += complex(amp[k]) * torch.polar(torch.ones_like(arg), arg)
    return (acc / math.sqrt(2.0 * n_waves)).to(torch.complex64)


@dataclass
class RadarPairScene:
    """Reference/secondary burst pair for radar-grid coregistration."""
    name: str
    seed: int
    ref: Acquisition
    sec: Acquisition
    lat: object  # float64 [L, S] of the reference grid
    lon: object
    hgt: object
    ref_slc: object  # complex64 [L, S], TOPS-modulated
    sec_slc: object
    rowlook: int
    collook: int
    alpha: float
    win: int = 5
    n_win: int = 32
    extra: dict = field(default_factory=dict)

    @property
    def burst_pixels(self):
        return int(self.ref_slc.shape[0]) * int(self.ref_slc.shape[1])


def make_radar_pair(config="c1", seed=20261203, device="cpu", baseline=150.0, coherence=0.7,
                    lines=None, samples=None, defo_amp=0.03, defo_sigma=5000.0):
    """Radar-grid burst pair: float64 lat/lon/height rasters of the
    reference grid, a secondary with a perpendicular baseline, a band-limited
    reflectivity seen by both, a Gaussian deformation (phase 4 pi d / lambda)
    and coherence ``coherence`` against white noise."""
    import torch
    L, S, rl, cl, al, hmax, kt = CONFIGS[config]
    L = int(lines or L)
    S = int(samples or S)
    t_c = ORBIT_T0 + 50.0
    orbit_ref = make_orbit(t_c=t_c)
    off = secondary_offset(orbit_ref, t_c, NEAR_RANGE + S * RANGE_SPACING / 2, baseline)
    orbit_sec = make_orbit(t_c=t_c, offset=off)
    radar = make_radar(L, S, hmin=-100.0, hmax=hmax + 100.0)
    t_start = t_c - L * AZIMUTH_INTERVAL / 2
    fm, dc = tops_tables(radar, t_c, kt)
    burst = burst_meta(t_start, L, S, margin_l=4, margin_s=4)
    ref = Acquisition(radar=radar, orbit=orbit_ref, fm=fm, dc=dc, bursts=[burst])
    sec = Acquisition(radar=radar, orbit=orbit_sec, fm=fm.copy(), dc=dc.copy(), bursts=[burst])
    hfun = lambda la, lo: fbm_height(la, lo, seed, hmax)
    lat, lon, hgt = rdr2geo_grid(orbit_ref, radar, burst, hfun, device=device)
    slat, slon, _ = rdr2geo_grid(orbit_sec, radar, burst, hfun, device=device)
    lat0, lon0 = float(lat[L // 2, S // 2]), float(lon[L // 2, S // 2])
    f_ref = reflectivity(lat, lon, seed, lat0, lon0)
    f_sec = reflectivity(slat, slon, seed, lat0, lon0)
    # deformation seen by the secondary: 2-D Gaussian in ground metres
    north = (slat - lat0) * (math.pi / 180.0 * RA)
    east = (slon - lon0) * (math.pi / 180.0 * RA * math.cos(math.radians(lat0)))
    dphi = (4 * math.pi / WAVELENGTH) * defo_amp * torch.exp(-(north ** 2 + east ** 2) / (2 * defo_sigma ** 2))
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    noise = speckle(L, S, gen, device)
    s_sec = coherence * f_sec * torch.polar(torch.ones_like(dphi), dphi).to(torch.complex64) + \
        math.sqrt(1 - coherence ** 2) * noise
    ref_slc = tops_modulate(f_ref, ref, burst).contiguous()
    sec_slc = tops_modulate(s_sec.to(torch.complex64), sec, burst).contiguous()
    return RadarPairScene(name=config, seed=seed, ref=ref, sec=sec, lat=lat, lon=lon, hgt=hgt, ref_slc=ref_slc,
                          sec_slc=sec_slc, rowlook=rl, collook=cl, alpha=al, extra={"hmax": hmax})


@dataclass
class RefineStack:
    """Bursts for coherence-maximising coregistration refinement: one radar
    grid geometry shared by every burst, independent speckle, true offset
    polynomials and height errors per burst."""
    sec_plans: list
    ref: object      # complex64 [n, L, S]
    sec: object      # complex64 [n, lines, samples] (secondary bursts)
    az0: object      # float32 [n, L, S] geometric offsets (from the heights in the rasters)
    rg0: object
    daz_dh: object   # float32 [n, L, S]
    drg_dh: object
    params_true: object  # float32 [n, 6]
    dh_true: object      # float32 [n, L, S]
    rowlook: int
    collook: int
    coherence: float
    sec_acq: object = None   # the secondary Acquisition (radar, orbit, TOPS tables)
    ref_acq: object = None   # the reference Acquisition
    geometry: object = None  # (lat, lon, hgt) float64 rasters of the burst, kept when asked for
    margin: int = 0          # reference grid = burst minus this many pixels on every side


def gaussian_smooth(x, sigma):
    """Separable Gaussian smoothing of [n, L, S] float32 (torch, edge padding)."""
    import torch
    r = int(3 * sigma)
    t = torch.arange(-r, r + 1, dtype=torch.float32, device=x.device)
    k = torch.exp(-0.5 * (t / sigma) ** 2)
    k = k / k.sum()
    y = x[:, None]
    y = torch.nn.functional.pad(y, (r, r, 0, 0), mode="replicate")
    y = torch.nn.functional.conv2d(y, k.view(1, 1, 1, -1))
    y = torch.nn.functional.pad(y, (0, 0, r, r), mode="replicate")
    y = torch.nn.functional.conv2d(y, k.view(1, 1, -1, 1))
    return y[:, 0]


def make_refine_stack(n_bursts=8, config="c1", seed=20261203 + 3000, device="cuda", param_sigma=0.05,
                      dh_sigma=10.0, dh_smooth=31.0, coherence=0.7, lines=None, samples=None, keep_geometry=False,
                      margin=0):
    """Refinement stack (GPU).  The geometry is that of ``make_radar_pair``
    (float64 lat/lon/height rasters of the reference grid, secondary orbit
    with a 150 m baseline).  Per burst: the secondary is white speckle W,
    TOPS-modulated so that deramping returns W; the true secondary coordinates
    are the geometric offsets plus an offset polynomial params_true ~ N(0,
    param_sigma) (samples) plus the height sensitivities times dh_true, a
    N(0, 1) field smoothed by a ``dh_smooth``-pixel Gaussian and scaled to
    ``dh_sigma`` metres rms; the reference is coherence * (secondary
    resampled there with the 8-tap sinc) + sqrt(1 - coherence^2) * noise.
    Refinement from zero should move toward (params_true, dh_true).
    ``margin`` > 0 makes the reference grid the burst minus ``margin``
    pixels on every side (offsets shifted accordingly), so that no pixel's
    8 x 8 support reaches the secondary burst's edge."""
    import torch

    from . import kernels, plan as _plan
    sc = make_radar_pair(config, seed=seed, device=device, lines=lines, samples=samples)
    sp = _plan.burst_plan(sc.sec.radar, sc.sec.orbit, sc.sec.fm, sc.sec.dc, sc.sec.bursts[0], None)
    rp = _plan.burst_plan(sc.ref.radar, sc.ref.orbit, sc.ref.fm, sc.ref.dc, sc.ref.bursts[0], None)
    az0, rg0, daz, drg = kernels.geo2rdr_offsets_dh(sp, rp, sc.lat, sc.lon, sc.hgt)
    m = int(margin)
    if m > 0:
        az0 = (az0[m:-m, m:-m] + m).contiguous()
        rg0 = (rg0[m:-m, m:-m] + m).contiguous()
        daz = daz[m:-m, m:-m].contiguous()
        drg = drg[m:-m, m:-m].contiguous()
    L, S = az0.shape
    geometry = (sc.lat, sc.lon, sc.hgt) if keep_geometry else None
    sc.lat = sc.lon = sc.hgt = None
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    params = torch.tensor(rng.normal(0.0, param_sigma, (n_bursts, 6)), dtype=torch.float32, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed + 2)
    dh = gaussian_smooth(torch.randn((n_bursts, L, S), generator=gen, device=device), dh_smooth)
    dh = dh * (dh_sigma / dh.std())
    rows = torch.arange(L, dtype=torch.float32, device=device)[:, None]
    cols = torch.arange(S, dtype=torch.float32, device=device)[None, :]
    xa, xr = (rows - 0.5 * L) / L, (cols - 0.5 * S) / S
    # secondary deramp phase of every sample, -pi kt (eta - etaref)^2 (the
    # resampler multiplies by exp(i phase) before interpolating)
    kt, etaref, eta = tops_coefficients(sc.sec, sc.sec.bursts[0])
    kt_t = torch.tensor(kt, dtype=torch.float64, device=device)[None, :]
    er_t = torch.tensor(etaref, dtype=torch.float64, device=device)[None, :]
    eta_t = torch.tensor(eta, dtype=torch.float64, device=device)[:, None]
    phase = -math.pi * kt_t * (eta_t - er_t) ** 2
    rot = torch.polar(torch.ones_like(phase), -phase).to(torch.complex64)
    del phase
    ref = torch.empty((n_bursts, L, S), dtype=torch.complex64, device=device)
    Ls, Ss = rot.shape
    sec = torch.empty((n_bursts, Ls, Ss), dtype=torch.complex64, device=device)
    for b in range(n_bursts):
        w = speckle(Ls, Ss, gen, device)
        sec[b] = w * rot
        p = params[b]
        az_t = (az0 + p[0] + p[1] * xa + p[2] * xr + daz * dh[b]).contiguous()
        rg_t = (rg0 + p[3] + p[4] * xa + p[5] * xr + drg * dh[b]).contiguous()
        s_true = kernels.resample(sp, sec[b], az_t, rg_t)
        ref[b] = coherence * s_true + math.sqrt(1 - coherence ** 2) * speckle(L, S, gen, device)
    stack = RefineStack(sec_plans=[sp] * n_bursts, ref=ref, sec=sec,
                        az0=az0.expand(n_bursts, L, S).contiguous(), rg0=rg0.expand(n_bursts, L, S).contiguous(),
                        daz_dh=daz.expand(n_bursts, L, S).contiguous(), drg_dh=drg.expand(n_bursts, L, S).contiguous(),
                        params_true=params, dh_true=dh.contiguous(), rowlook=sc.rowlook, collook=sc.collook,
                        coherence=coherence, sec_acq=sc.sec, ref_acq=sc.ref, geometry=geometry, margin=m)
    return stack
