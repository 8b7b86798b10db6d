"""interfere() (s1proc/interfere.py:536-704) end to end on geocoded burst
files of two dates (two subswaths, two bursts each, written in the .gslc
format): the multilooked RSC, the stitched interferogram of the date pair,
the burst files removed; the frame against the float64 oracle's crossmul of
every matched burst pair (oracle/crossmul.py) stitched by the oracle
(oracle/stitch.py), itself pinned to the reference's Python."""
import os

import numpy as np
import pytest

from helpers import phase_rms
from oracle import crossmul as ox
from oracle import stitch as ost
from sentinel_gpu_processor_b200 import formats, interfere as I

pytestmark = pytest.mark.gpu

NROW0, NCOL0 = 160, 320
BOXES = {1: [(10, 4, 150, 60), (12, 50, 148, 108), (9, 100, 151, 158)], 2: [(140, 0, 310, 62), (141, 52, 309, 110)]}


def _write_date(d, date, uid, rng, field, shift):
    files = []
    for sw, boxes in BOXES.items():
        for k, (l, t, r, b) in enumerate(boxes):
            l2, t2, r2, b2 = l + shift, t + shift, r + shift, b + shift
            z = field[t2:b2, l2:r2] + 0.3 * (rng.standard_normal((b2 - t2, r2 - l2)) +
                                             1j * rng.standard_normal((b2 - t2, r2 - l2)))
            z = z.astype(np.complex64)
            z[:, :3] = 0
            f = os.path.join(d, f"{date}_S1A_{uid}_iw{sw}_burst_{k}.gslc")
            formats.write_raster(f, formats.make_header(NROW0, NCOL0, l2, t2, r2, b2), z)
            files.append(f)
    return files


def test_interfere_matches_oracle(cuda, tmp_path):
    rng = np.random.default_rng(3)
    yy, xx = np.mgrid[0:NROW0, 0:NCOL0]
    field = np.exp(1j * (0.04 * xx + 0.02 * yy))
    slc = tmp_path / "slc"
    ifgs = tmp_path / "igrams"
    slc.mkdir()
    ifgs.mkdir()
    _write_date(str(slc), "20200101", "AAAA", rng, field, 0)
    _write_date(str(slc), "20200113", "BBBB", rng, field * np.exp(1j * 0.01 * yy), 1)
    rsc = formats.Rsc(NROW0, NCOL0, 36.0, 14.0, -1.0 / 7200, 1.0 / 7200)
    formats.write_rsc(str(tmp_path / "dem.rsc"), rsc)
    (ifgs / "pairs.txt").write_text("20200101 20200113\n")
    rl, cl = 2, 4
    # the reference burst files, as interfere() pairs them (before they are removed)
    tasks = I.burst_pair_tasks(sorted(str(p) for p in slc.glob("20200101*.gslc")),
                               sorted(str(p) for p in slc.glob("20200113*.gslc")), str(ifgs))
    want_bursts = []
    for f1, f2, out in tasks:
        h1, d1 = formats.read_raster(f1)
        h2, d2 = formats.read_raster(f2)
        hd, data = ox.crossmul_pair(h1, d1, h2, d2, rl, cl)
        w = os.path.basename(out).split("_")
        want_bursts.append((hd, data, int(w[3][2]), (w[1] + w[2], w[7] + w[8])))
    groups = {}
    want = ost.stitch([(h, d, sw, groups.setdefault(g, len(groups))) for h, d, sw, g in want_bursts],
                      NROW0 // rl, NCOL0 // cl)
    ok, failed = I.interfere("pairs.txt", str(slc), str(tmp_path / "dem.rsc"), str(tmp_path / "small" / "dem.rsc"),
                             str(ifgs), rl, cl)
    assert (ok, failed) == (len(tasks), 0)
    out = ifgs / "20200101_20200113.int"
    got = np.fromfile(str(out), dtype=np.complex64).reshape(NROW0 // rl, NCOL0 // cl)
    np.testing.assert_array_equal(np.abs(got) > 0, np.abs(want) > 0)
    assert np.abs(got - want).max() < 1e-5 * np.abs(want).max()
    assert phase_rms(got, want) < 1e-5
    assert not any(os.path.exists(t[2]) for t in tasks)
    small = formats.read_rsc(str(tmp_path / "small" / "dem.rsc"))
    assert (small.nlat, small.nlon) == (NROW0 // rl, NCOL0 // cl)
    # a second call finds the interferogram and does nothing
    assert I.interfere("pairs.txt", str(slc), str(tmp_path / "dem.rsc"), str(tmp_path / "small" / "dem.rsc"),
                       str(ifgs), rl, cl) == (0, 0)
