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


def write_cint16_tiff(path, arr, rows_per_strip=None, tile=None, big=False, byteorder="<", two_samples=False,
                      compression=1):
    """Minimal TIFF writer for tests: one directory, int16 [H, W, 2] (re, im)
    samples as CInt16 (BitsPerSample 32, SampleFormat 5) or, with
    ``two_samples``, two int16 samples per pixel.  Image blocks first, then
    the out-of-line tag values, then the directory (so the reader must follow
    the directory offset).  Strips of ``rows_per_strip`` rows, or tiles of
    ``tile`` = (width, height) padded with zeros at the edges."""
    import struct as st
    H, W, _ = arr.shape
    bo = byteorder
    a = np.ascontiguousarray(arr, dtype=np.int16).astype(bo + "i2")
    hdr = 16 if big else 8
    blocks = []
    if tile is None:
        rps = rows_per_strip or H
        for r in range(0, H, rps):
            blocks.append(a[r:r + rps].tobytes())
    else:
        tw, th = tile
        for ty in range(0, H, th):
            for tx in range(0, W, tw):
                t = np.zeros((th, tw, 2), dtype=bo + "i2")
                part = a[ty:ty + th, tx:tx + tw]
                t[:part.shape[0], :part.shape[1]] = part
                blocks.append(t.tobytes())
    offs, pos = [], hdr
    for b in blocks:
        offs.append(pos)
        pos += len(b)
    counts = [len(b) for b in blocks]
    lng = 16 if big else 4  # LONG8 or LONG for offset tables
    tags = {256: (4, [W]), 257: (4, [H]), 259: (3, [compression])}
    if two_samples:
        tags.update({258: (3, [16, 16]), 277: (3, [2]), 339: (3, [2, 2]), 284: (3, [1])})
    else:
        tags.update({258: (3, [32]), 277: (3, [1]), 339: (3, [5])})
    if tile is None:
        tags.update({273: (lng, offs), 278: (4, [rows_per_strip or H]), 279: (lng, counts)})
    else:
        tags.update({322: (3, [tile[0]]), 323: (3, [tile[1]]), 324: (lng, offs), 325: (lng, counts)})
    letter = {3: "H", 4: "I", 16: "Q"}
    size = {3: 2, 4: 4, 16: 8}
    inline = 8 if big else 4
    extra = b""
    entries = []
    for tag in sorted(tags):
        typ, vals = tags[tag]
        raw = st.pack(bo + letter[typ] * len(vals), *vals)
        if len(raw) <= inline:
            val = raw.ljust(inline, b"\0")
        else:
            val = st.pack(bo + ("Q" if big else "I"), pos + len(extra))
            extra += raw
        entries.append(st.pack(bo + ("HHQ" if big else "HHI"), tag, typ, len(vals)) + val)
    ifd_off = pos + len(extra)
    if big:
        head = st.pack(bo + "2sHHHQ", b"II" if bo == "<" else b"MM", 43, 8, 0, ifd_off)
        ifd = st.pack(bo + "Q", len(entries)) + b"".join(entries) + st.pack(bo + "Q", 0)
    else:
        head = st.pack(bo + "2sHI", b"II" if bo == "<" else b"MM", 42, ifd_off)
        ifd = st.pack(bo + "H", len(entries)) + b"".join(entries) + st.pack(bo + "I", 0)
    with open(path, "wb") as f:
        f.write(head + b"".join(blocks) + extra + ifd)
