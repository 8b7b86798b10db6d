"""s1proc file formats: cropped rasters with a 64 x int32 header, RSC grids,
orbit/FM-rate/Doppler text files and the per-subswath SQLite parameter DB.

These are the formats the reference executables read and write:
  * raster header ``[nrow0, ncol0, left, top, right, bottom, 0...]`` +
    row-major payload (``csrc/include/sario.hpp:14, 108-123``;
    ``s1proc/sario.py:19, 85-97``)
  * RSC text ``WIDTH FILE_LENGTH X_FIRST Y_FIRST X_STEP Y_STEP``
    (``csrc/src/sario.cu:12-60``; writer ``s1proc/geocoordinates.py:87-98``)
  * orbit ASCII: count line, then ``t x y z vx vy vz 0 0 0`` per line
    (``s1proc/sentinel_roidb.py:605-622``; reader ``csrc/src/orbit.cu:147-168``)
  * FM-rate / Doppler-centroid text: count line, then ``time t0 c0 c1 c2``
    (``s1proc/sentinel_roidb.py:733-786``; reader ``csrc/src/sario.cu:80-103``)
  * SQLite table ``file(t1key, name, value, units, type, comments)``
    (``s1proc/sql_mod.py:5-19``; reader ``csrc/src/sql_mod.cpp:17-85``) with
    the keys read at ``csrc/src/geo2rdr.cu:333-376``.
"""
from __future__ import annotations

import os
import sqlite3
from dataclasses import dataclass

import numpy as np

NHEADER = 64


# ----------------------------------------------------------------------------
# Rasters
# ----------------------------------------------------------------------------

def make_header(nrow0, ncol0, left, top, right, bottom):
    h = np.zeros(NHEADER, dtype=np.int32)
    h[:6] = [nrow0, ncol0, left, top, right, bottom]
    return h


def write_raster(path, header, data):
    """save_binary with header (sario.hpp:108-123)."""
    with open(path, "wb") as f:
        np.asarray(header, dtype=np.int32).tofile(f)
        np.ascontiguousarray(data).tofile(f)


def read_header(path):
    return np.fromfile(path, dtype=np.int32, count=NHEADER)


def read_raster(path, dtype=np.complex64):
    """Cropped raster -> (header, data [bottom-top, right-left])."""
    with open(path, "rb") as f:
        h = np.fromfile(f, dtype=np.int32, count=NHEADER)
        nrow = int(h[5]) - int(h[3])
        ncol = int(h[4]) - int(h[2])
        d = np.fromfile(f, dtype=dtype, count=nrow * ncol)
    if d.size != nrow * ncol:
        raise IOError(f"{path}: truncated raster ({d.size} of {nrow * ncol} elements)")
    return h, d.reshape(nrow, ncol)


# ----------------------------------------------------------------------------
# RSC grid
# ----------------------------------------------------------------------------

@dataclass
class Rsc:
    nlat: int
    nlon: int
    latmax: float
    lonmin: float
    dlat: float
    dlon: float

    def take_look(self, latlook, lonlook):
        """geocoordinates.py:153-161."""
        return Rsc(nlat=self.nlat // latlook, nlon=self.nlon // lonlook,
                   latmax=self.latmax + self.dlat * (latlook - 1.0) / 2,
                   lonmin=self.lonmin + self.dlon * (lonlook - 1.0) / 2,
                   dlat=self.dlat * latlook, dlon=self.dlon * lonlook)


def write_rsc(path, rsc: Rsc):
    """Format of geocoordinates.py:87-98 (14 decimals)."""
    with open(path, "w") as f:
        f.write("{0: <16}{1:d}\n".format("WIDTH", rsc.nlon))
        f.write("{0: <16}{1:d}\n".format("FILE_LENGTH", rsc.nlat))
        f.write("{0: <16}{1:.14f}\n".format("X_FIRST", rsc.lonmin))
        f.write("{0: <16}{1:.14f}\n".format("Y_FIRST", rsc.latmax))
        f.write("{0: <16}{1:.14f}\n".format("X_STEP", rsc.dlon))
        f.write("{0: <16}{1:.14f}\n".format("Y_STEP", rsc.dlat))
        f.write("{0: <16}{1}\n".format("Z_OFFSET", 0))
        f.write("{0: <16}{1}\n".format("Z_SCALE", 1))
        f.write("{0: <16}{1}".format("PROJECTION", "LATLON"))


def read_rsc(path) -> Rsc:
    """readrsc, sario.cu:12-60."""
    vals = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2:
                vals[parts[0]] = parts[1]
    return Rsc(nlat=int(vals["FILE_LENGTH"]), nlon=int(vals["WIDTH"]),
               latmax=float(vals["Y_FIRST"]), lonmin=float(vals["X_FIRST"]),
               dlat=float(vals["Y_STEP"]), dlon=float(vals["X_STEP"]))


def rsc_roundtrip(rsc: Rsc) -> Rsc:
    """The values a reader gets back after ``write_rsc`` (14-decimal text)."""
    f = lambda v: float("{0:.14f}".format(v))
    return Rsc(rsc.nlat, rsc.nlon, f(rsc.latmax), f(rsc.lonmin), f(rsc.dlat), f(rsc.dlon))


# ----------------------------------------------------------------------------
# Orbit and polynomial text files
# ----------------------------------------------------------------------------

def write_orbit_ascii(path, tt, xx, vv):
    tt = np.asarray(tt, dtype=np.float64)
    xx = np.asarray(xx, dtype=np.float64).reshape(-1, 3)
    vv = np.asarray(vv, dtype=np.float64).reshape(-1, 3)
    with open(path, "w") as f:
        f.write(f"{len(tt)}\n")
        for i in range(len(tt)):
            f.write(" ".join(repr(float(v)) for v in (tt[i], *xx[i], *vv[i])) + " 0.0 0.0 0.0\n")


def read_orbit_ascii(path):
    with open(path) as f:
        n = int(f.readline().split()[0])
        rows = [list(map(float, f.readline().split()[:7])) for _ in range(n)]
    a = np.asarray(rows, dtype=np.float64)
    return a[:, 0].copy(), a[:, 1:4].copy(), a[:, 4:7].copy()


def write_poly(path, table):
    """table [n, 5] columns (time, t0, c0, c1, c2)."""
    table = np.asarray(table, dtype=np.float64)
    with open(path, "w") as f:
        f.write(f"{len(table)}\n")
        for row in table:
            f.write(" ".join(repr(float(v)) for v in row) + "\n")


def read_poly(path):
    with open(path) as f:
        n = int(f.readline().split()[0])
        rows = [list(map(float, f.readline().split()[:5])) for _ in range(n)]
    return np.asarray(rows, dtype=np.float64).reshape(n, 5)


# ----------------------------------------------------------------------------
# Parameter DB
# ----------------------------------------------------------------------------

def write_db(path, params: dict):
    """Create the ``file`` table (sql_mod.py:5-19) and store ``params``.

    Every column is filled: the reference reader converts all five columns to
    ``std::string`` (sql_mod.cpp:49-58), so a NULL would be dereferenced.
    """
    if os.path.exists(path):
        os.remove(path)
    con = sqlite3.connect(path)
    c = con.cursor()
    c.execute("create table file (t1key INTEGER PRIMARY KEY, name TEXT unique, value TEXT, "
              "units text, type text, comments text);")
    for k, v in params.items():
        if isinstance(v, float):
            sv, ty = repr(v), "real*8"
        elif isinstance(v, (int, np.integer)):
            sv, ty = str(int(v)), "int*4"
        else:
            sv, ty = str(v), "CHAR"
        c.execute("insert into file (name, value, units, type, comments) values (?, ?, ?, ?, ?)",
                  (k, sv, "-", ty, k))
    con.commit()
    con.close()


def read_db(path) -> dict:
    con = sqlite3.connect(path)
    out = {name: value for name, value in con.execute("select name, value from file")}
    con.close()
    return out
