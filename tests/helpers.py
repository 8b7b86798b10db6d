"""Shared test helpers: scene -> oracle records, error metrics."""
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
