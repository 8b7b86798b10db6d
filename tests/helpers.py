"""Shared test helpers: scene -> oracle records, golden-fixture records, error metrics."""
import os
from types import SimpleNamespace

import numpy as np

from oracle import geo2rdr as og2


def oracle_radar(r):
    return og2.Radar(**{k: getattr(r, k) for k in og2.Radar.__dataclass_fields__})


def oracle_burst(b):
    return og2.BurstMeta(**{k: getattr(b, k) for k in og2.BurstMeta.__dataclass_fields__})


def oracle_rsc(r):
    return og2.Rsc(nlat=r.nlat, nlon=r.nlon, latmax=r.latmax, lonmin=r.lonmin, dlat=r.dlat, dlon=r.dlon)


def phase_rms(a, b, mask=None):
    """RMS of the wrapped phase difference angle(a * conj(b)) over ``mask`` (rad)."""
    a = np.asarray(a).astype(np.complex128)
    b = np.asarray(b).astype(np.complex128)
    m = (np.abs(a) > 0) & (np.abs(b) > 0)
    if mask is not None:
        m &= mask
    d = np.angle(a[m] * np.conj(b[m]))
    return float(np.sqrt(np.mean(d * d))) if d.size else 0.0


def rel_err(a, b, mask=None):
    """max |a - b| / max |b| (complex or real)."""
    a = np.asarray(a).astype(np.complex128)
    b = np.asarray(b).astype(np.complex128)
    if mask is not None:
        a, b = a[mask], b[mask]
    den = np.abs(b).max() if b.size else 1.0
    return float(np.abs(a - b).max() / max(den, 1e-30)) if b.size else 0.0


GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_chain_tiny.npz")


def golden_acq(z, prefix):
    """Acquisition record (radar, bursts, orbit, FM/DC tables) of the golden fixture."""
    r = z[prefix + "radar"]
    b = z[prefix + "burst"]
    radar = og2.Radar(samples_per_burst=int(r[0]), lines_per_burst=int(r[1]), prf=r[2], wvl=r[3], hmin=r[4],
                      hmax=r[5], range_sampling_rate=r[6], slant_range_time=r[7], azimuth_steering_rate=r[8],
                      azimuth_time_interval=r[9], radar_frequency=r[10])
    burst = og2.BurstMeta(azimuth_time=b[0], first_valid_line=int(b[1]), last_valid_line=int(b[2]),
                          first_valid_sample=int(b[3]), last_valid_sample=int(b[4]))
    orbit = (z[prefix + "tt"], z[prefix + "xx"], z[prefix + "vv"])
    return SimpleNamespace(radar=radar, bursts=[burst], orbit=orbit, fm=z[prefix + "fm"], dc=z[prefix + "dc"])


def golden_rsc(z):
    r = z["rsc"]
    return og2.Rsc(nlat=int(r[0]), nlon=int(r[1]), latmax=r[2], lonmin=r[3], dlat=r[4], dlon=r[5])
