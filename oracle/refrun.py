"""Run the reference executables (built by ``oracle/build_ref.py``) on
synthetic inputs written in the reference's own file formats.

Test infrastructure only (see ``oracle/__init__.py``): used by the GPU
parity tests, by ``tests/golden/make_golden.py`` and by the reference arm of
``bench.py``.  The executables run on a CUDA GPU.
"""
from __future__ import annotations

import os
import subprocess
import time

import numpy as np

from sentinel_gpu_processor_b200 import formats

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "bin")


def available():
    return all(os.path.exists(os.path.join(BIN, b)) for b in ("geo2rdr", "crossmul_daemon", "goldstein"))


def write_dem(workdir, rsc, dem, name="dem"):
    rscf = os.path.join(workdir, name + ".rsc")
    demf = os.path.join(workdir, name + ".dem")
    formats.write_rsc(rscf, rsc)
    np.ascontiguousarray(dem, dtype=np.int16).tofile(demf)
    return rscf, demf


def write_geo2rdr_inputs(workdir, tag, acq, slcs, rscf, demf):
    """DB + orbit/FM/DC text + raw SLC for one geo2rdr run (geo2rdr.cu:333-384).

    ``slcs``: list of complex64 [L, S] bursts (all the same size), written
    back to back as the reference's ``slc_file``.
    """
    r = acq.radar
    orbf = os.path.join(workdir, tag + "_orb.txt")
    fmf = os.path.join(workdir, tag + "_fm.txt")
    dcf = os.path.join(workdir, tag + "_dc.txt")
    slcf = os.path.join(workdir, tag + ".slc")
    formats.write_orbit_ascii(orbf, *acq.orbit)
    formats.write_poly(fmf, acq.fm)
    formats.write_poly(dcf, acq.dc)
    with open(slcf, "wb") as f:
        for s in slcs:
            np.ascontiguousarray(s, dtype=np.complex64).tofile(f)
    params = {
        "demfile": demf, "rscfile": rscf,
        "samplesPerBurst": int(r.samples_per_burst), "linesPerBurst": int(r.lines_per_burst),
        "azimuthBursts": len(acq.bursts), "prf": float(r.prf), "wvl": float(r.wvl),
        "hmin": float(r.hmin), "hmax": float(r.hmax), "rangeSamplingRate": float(r.range_sampling_rate),
        "slantRangeTime": float(r.slant_range_time), "azimuthSteeringRate": float(r.azimuth_steering_rate),
        "azimuthTimeInterval": float(r.azimuth_time_interval), "radarFrequency": float(r.radar_frequency),
        "orbinfo": orbf, "fmrateinfo": fmf, "dcinfo": dcf, "slc_file": slcf,
    }
    for i, b in enumerate(acq.bursts):
        params[f"azimuthTimeSeconds{i + 1}"] = float(b.azimuth_time)
        params[f"firstValidLine{i + 1}"] = int(b.first_valid_line)
        params[f"lastValidLine{i + 1}"] = int(b.last_valid_line)
        params[f"firstValidSample{i + 1}"] = int(b.first_valid_sample)
        params[f"lastValidSample{i + 1}"] = int(b.last_valid_sample)
    db = os.path.join(workdir, tag + ".db")
    formats.write_db(db, params)
    return db


def run(cmd, log=None, timeout=1800):
    t0 = time.perf_counter()
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=timeout)
    dt = time.perf_counter() - t0
    if log is not None:
        log.append({"cmd": cmd, "rc": r.returncode, "seconds": dt, "stdout": r.stdout[-2000:],
                    "stderr": r.stderr[-2000:]})
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(cmd[0])} failed ({r.returncode}): {r.stderr[-800:]}")
    return dt, r.stdout


def geo2rdr(db, outprefix, nbursts, log=None):
    """Run the reference geo2rdr; returns ([(header, data) or None per burst], seconds)."""
    dt, _ = run([os.path.join(BIN, "geo2rdr"), db, outprefix], log)
    outs = []
    for i in range(nbursts):
        f = f"{outprefix}_burst_{i}.gslc"
        outs.append(formats.read_raster(f) if os.path.exists(f) else None)
    return outs, dt


def crossmul_daemon(tasks, tasks_file, rowlook, collook, out_float=False, manual=True, log=None):
    """Run the reference crossmul_daemon on [(ref, sec, out)] tasks; returns (stdout, seconds)."""
    with open(tasks_file, "w") as f:
        for t in tasks:
            f.write(f"{t[0]} {t[1]} {t[2]}\n")
    cmd = [os.path.join(BIN, "crossmul_daemon"), "--rowlook", str(rowlook), "--collook", str(collook),
           "--tasks-file", tasks_file]
    if manual:
        cmd += ["--io-workers", "1", "--cpu-workers", "1", "--gpu-workers", "1", "--streams-per-gpu", "1",
                "--max-slots", "1"]
    if out_float:
        cmd.append("--out-float")
    dt, out = run(cmd, log)
    return out, dt


def goldstein(infile, nrow, ncol, n_win, alpha, log=None):
    """Run the reference goldstein on one ``.int`` file -> (filtered complex64, seconds).

    With a single ``.int`` input the executable writes ``filtered.int`` into
    its working directory (goldstein.cu:471-474); it is run from the input's
    directory.
    """
    wd = os.path.dirname(os.path.abspath(infile))
    cmd = [os.path.join(BIN, "goldstein"), os.path.abspath(infile), str(nrow), str(ncol), str(n_win), repr(float(alpha))]
    t0 = time.perf_counter()
    r = subprocess.run(cmd, cwd=wd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=1800)
    dt = time.perf_counter() - t0
    if log is not None:
        log.append({"cmd": cmd, "rc": r.returncode, "seconds": dt})
    if r.returncode != 0:
        raise RuntimeError(f"goldstein failed: {r.stderr[-800:]}")
    out = np.fromfile(os.path.join(wd, "filtered.int"), dtype=np.complex64).reshape(nrow, ncol)
    return out, dt


def geo2rdr_buffers_safe(acq, rsc):
    """True when the reference geo2rdr's DEM/output buffers fit every burst window.

    geo2rdr.cu:408-423 sizes its host DEM buffer and device output buffer as
    ``int((latmin - latmax)/dlat + 1) x int((lonmax - lonmin)/dlon + 1)`` (max
    over bursts), while each burst's window (569-586) truncates its two ends
    separately and can be one row or column larger.  Then the host DEM read
    and the device output of ``reproject`` overrun their allocations.  The
    reference is only run on inputs for which this check passes.
    """
    from oracle import geo2rdr as og2
    r = og2.Radar(**{k: getattr(acq.radar, k) for k in og2.Radar.__dataclass_fields__})
    orsc = og2.Rsc(nlat=rsc.nlat, nlon=rsc.nlon, latmax=rsc.latmax, lonmin=rsc.lonmin, dlat=rsc.dlat, dlon=rsc.dlon)
    nrow_buf = ncol_buf = 0
    wins = []
    for b in acq.bursts:
        bm = og2.BurstMeta(**{k: getattr(b, k) for k in og2.BurstMeta.__dataclass_fields__})
        latmin, latmax, lonmin, lonmax = og2.burst_latlon_box(r, acq.orbit, bm)
        nrow_buf = max(nrow_buf, int((latmin - latmax) / rsc.dlat + 1))
        ncol_buf = max(ncol_buf, int((lonmax - lonmin) / rsc.dlon + 1))
        wins.append(og2.dem_window((latmin, latmax, lonmin, lonmax), orsc))
    # both buffers are flat: what must fit is the element count
    return all(w.nrow * w.ncol <= nrow_buf * ncol_buf for w in wins)


def footprint_boxes(acq):
    """Footprint box (latmin, latmax, lonmin, lonmax) of every burst of one
    geo2rdr run, from the oracle's restatement of bounds (geo2rdr.cu:387-400)."""
    from oracle import geo2rdr as og2
    r = og2.Radar(**{k: getattr(acq.radar, k) for k in og2.Radar.__dataclass_fields__})
    return [tuple(float(v) for v in og2.burst_latlon_box(
        r, acq.orbit, og2.BurstMeta(**{k: getattr(b, k) for k in og2.BurstMeta.__dataclass_fields__})))
        for b in acq.bursts]


def make_reference_safe(sc, acqs=None):
    """Return ``sc`` on a DEM grid where the reference geo2rdr stays inside its
    buffers for every acquisition in ``acqs`` (default: all of the scene's),
    moved by a fraction of a pixel if needed (synth.reference_safe_rsc, fed
    with the oracle's footprint boxes); the DEM is regenerated there."""
    from sentinel_gpu_processor_b200 import synth
    acqs = list(sc.ref) + list(sc.sec) if acqs is None else list(acqs)
    rsc = synth.reference_safe_rsc(sc.rsc, [footprint_boxes(a) for a in acqs])
    out = synth.regrid(sc, rsc)
    if not all(geo2rdr_buffers_safe(a, out.rsc) for a in acqs):
        raise RuntimeError("reference buffer check disagrees with the grid search")
    return out
