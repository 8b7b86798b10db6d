"""Geocoding of TOPS bursts onto a DEM grid: the in-process equivalent of the
reference ``geo2rdr`` executable (csrc/src/geo2rdr.cu:316-651).

``geocode_burst`` = deramp -> zero-Doppler geocoding with bilinear
resampling, reramp and range phase -> crop to the non-zero rows, returning the
``.gslc`` header and data the executable would write.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, formats, kernels, plan as _plan


def plans_for(acq, rsc):
    """One s1b_burst_plan_t per burst of an acquisition (synth.Acquisition-like)."""
    return [_plan.burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, b, rsc) for b in acq.bursts]


def gslc_header(plan, first, last):
    """geo2rdr.cu:641-647."""
    return formats.make_header(plan.rsc_nlat, plan.rsc_nlon, plan.win_left, plan.win_top + first,
                               plan.win_right, plan.win_top + last)


def geocode_burst(plan, slc: torch.Tensor, dem: torch.Tensor, deramped: torch.Tensor | None = None,
                  out: torch.Tensor | None = None, sync: bool = True):
    """Deramp + geocode one burst (``slc`` complex64, or complex int16 as
    int16 [..., 2] straight from the measurement TIFF).

    Returns (header int32[64], data view [rows, ncol]) like the ``.gslc`` the
    reference writes, or None when it would skip the burst (empty window or no
    non-zero row).  With ``sync=False`` returns (full window output, rows
    tensor) without reading the row range back to the host.
    """
    if plan.nrow <= 0 or plan.ncol <= 0:
        return None
    flat = slc.reshape(-1, 2) if slc.dtype == torch.int16 else slc.reshape(-1)
    deramped = kernels.deramp(plan, flat, out=deramped)
    full, rows = kernels.geo2rdr(plan, dem, deramped, out=out)
    if not sync:
        return full, rows
    first, last = (int(v) for v in rows.cpu())
    if first >= plan.nrow or first == last or last < 0:
        return None
    return gslc_header(plan, first, last), full[first:last]


def geo2rdr_files(db_path, out_prefix, slc_path=None, stream=None, tiff=None):
    """File-level drop-in for ``geo2rdr dbname slcoutfile [slcinfile] [--stdin]``
    (geo2rdr.cu:704-734): reads the parameter DB and the files it names,
    writes ``<out>_burst_<i>.gslc``.  With ``stream`` (a binary file object,
    e.g. stdin) the bursts are read from it one after the other, every burst
    before its window is checked (geo2rdr.cu:551-557); a short read raises
    EOFError.  With ``tiff`` (an ``ingest.MeasurementTiff``) the bursts come
    straight from the measurement TIFF as complex int16 -- what the reference
    pipes in after widening (s1proc/sentinel_scene.py:164-207, 419-437) --
    read ahead into pinned buffers, only those with a DEM window.  Returns the
    list of written paths."""
    from types import SimpleNamespace
    p = formats.read_db(db_path)
    radar = SimpleNamespace(samples_per_burst=int(p["samplesPerBurst"]), lines_per_burst=int(p["linesPerBurst"]),
                            prf=float(p["prf"]), wvl=float(p["wvl"]), hmin=float(p["hmin"]), hmax=float(p["hmax"]),
                            range_sampling_rate=float(p["rangeSamplingRate"]),
                            slant_range_time=float(p["slantRangeTime"]),
                            azimuth_steering_rate=float(p["azimuthSteeringRate"]),
                            azimuth_time_interval=float(p["azimuthTimeInterval"]),
                            radar_frequency=float(p["radarFrequency"]))
    nb = int(p["azimuthBursts"])
    bursts = [SimpleNamespace(azimuth_time=float(p[f"azimuthTimeSeconds{i + 1}"]),
                              first_valid_line=int(p[f"firstValidLine{i + 1}"]),
                              last_valid_line=int(p[f"lastValidLine{i + 1}"]),
                              first_valid_sample=int(p[f"firstValidSample{i + 1}"]),
                              last_valid_sample=int(p[f"lastValidSample{i + 1}"])) for i in range(nb)]
    orbit = formats.read_orbit_ascii(p["orbinfo"])
    fm = formats.read_poly(p["fmrateinfo"])
    dc = formats.read_poly(p["dcinfo"])
    rsc = formats.read_rsc(p["rscfile"])
    dem = torch.from_numpy(np.fromfile(p["demfile"], dtype=np.int16).reshape(rsc.nlat, rsc.nlon)).cuda()
    src = slc_path or p.get("slc_file")
    L, S = radar.lines_per_burst, radar.samples_per_burst
    written = []
    if tiff is not None:
        from . import ingest
        if tiff.width != S:
            raise ValueError(f"TIFF width {tiff.width} != samplesPerBurst {S}")
        plans = [_plan.burst_plan(radar, orbit, fm, dc, b, rsc) for b in bursts]
        use = [i for i, pl in enumerate(plans) if pl.nrow > 0 and pl.ncol > 0]
        for i, slc in ingest.BurstStream(tiff, L, nb, indices=use):
            res = geocode_burst(plans[i], slc, dem)
            if res is None:
                continue
            hdr, data = res
            path = f"{out_prefix}_burst_{i}.gslc"
            formats.write_raster(path, hdr, data.cpu().numpy())
            written.append(path)
        return written
    for i, b in enumerate(bursts):
        if stream is not None:
            buf = stream.read(L * S * 8)
            if len(buf) != L * S * 8:
                raise EOFError(f"expected {L * S * 8} bytes from stdin, got {len(buf)}")
            raw = np.frombuffer(buf, dtype=np.complex64).copy()
        pl = _plan.burst_plan(radar, orbit, fm, dc, b, rsc)
        if pl.nrow <= 0 or pl.ncol <= 0:
            continue
        if stream is None:
            raw = np.fromfile(src, dtype=np.complex64, count=L * S, offset=i * L * S * 8)
            if raw.size != L * S:
                raise IOError(f"{src}: short read for burst {i}")
        res = geocode_burst(pl, torch.from_numpy(raw).cuda(), dem)
        if res is None:
            continue
        hdr, data = res
        path = f"{out_prefix}_burst_{i}.gslc"
        formats.write_raster(path, hdr, data.cpu().numpy())
        written.append(path)
    return written
