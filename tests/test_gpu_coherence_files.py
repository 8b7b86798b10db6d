"""s1proc's coherence and geometry call surfaces on the GPU
(sentinel_gpu_processor_b200/coherence.py, geometry.py) against the float64
oracle restatements: amplitude mosaics (.amp), .cc rasters, geodetic
conversions and line-of-sight vectors."""
import os

import numpy as np
import pytest

from oracle import coherence as oc
from oracle import geometry as og
from sentinel_gpu_processor_b200 import coherence as C, formats, geometry as G, synth

pytestmark = pytest.mark.gpu


def _crop(rng, nrow0, ncol0, left, top, right, bottom, zero_rows=0):
    d = (rng.standard_normal((bottom - top, right - left)) + 1j * rng.standard_normal((bottom - top, right - left)))
    d = d.astype(np.complex64)
    if zero_rows:
        d[:zero_rows] = 0
    return formats.make_header(nrow0, ncol0, left, top, right, bottom), d


@pytest.mark.parametrize("looks", [(4, 20), (2, 8), (1, 1)])
def test_multilook_mosaic_matches_oracle(cuda, tmp_path, looks):
    rl, cl = looks
    rng = np.random.default_rng(rl * 100 + cl)
    # two overlapping bursts of one date; the second fills only zeros of the first
    crops = [_crop(rng, 203, 517, 13, 7, 401, 130, zero_rows=5), _crop(rng, 203, 517, 37, 101, 509, 190)]
    paths = []
    for k, (h, d) in enumerate(crops):
        p = str(tmp_path / f"20200101_{k}.gslc")
        formats.write_raster(p, h, d)
        paths.append(p)
    out = str(tmp_path / "20200101.amp")
    C.multilook(paths, out, rl, cl)
    got = np.fromfile(out, dtype=np.float32).reshape(203 // rl, 517 // cl)
    want = oc.multilook(crops, rl, cl)
    np.testing.assert_array_equal(got > 0, want > 0)
    assert np.abs(got - want).max() <= 2e-6 * max(1.0, float(np.abs(want).max()))


def test_multilook_amp_and_coherence_files(cuda, tmp_path):
    rl, cl = 2, 4
    rng = np.random.default_rng(5)
    slc_dir, amp_dir, ifg_dir = (str(tmp_path / n) for n in ("slc", "amp", "ifg"))
    os.makedirs(slc_dir)
    os.makedirs(ifg_dir)
    for date in ("20200101", "20200113"):
        for k in range(2):
            h, d = _crop(rng, 64, 128, 8 * k, 4 * k, 100 + 8 * k, 50 + 4 * k)
            formats.write_raster(os.path.join(slc_dir, f"{date}_iw{k + 1}.gslc"), h, d)
    C.multilook_amp(slc_dir, amp_dir, rl, cl)
    a1 = np.fromfile(os.path.join(amp_dir, "20200101.amp"), dtype=np.float32).reshape(32, 32)
    a2 = np.fromfile(os.path.join(amp_dir, "20200113.amp"), dtype=np.float32).reshape(32, 32)
    ifg = (a1 * a2 * np.exp(1j * rng.uniform(-3, 3, a1.shape)) * rng.uniform(0.2, 1.2, a1.shape))
    ifg = ifg.astype(np.complex64)
    ifg.tofile(os.path.join(ifg_dir, "20200101_20200113.int"))
    C.coherence(ifg_dir, amp_dir, 32, 32, rl, cl)
    got = np.fromfile(os.path.join(ifg_dir, "20200101_20200113.cc"), dtype=np.float32).reshape(32, 64)
    prod, c = oc.coherence(ifg, a1, a2, seed=0)
    want = oc.cc_rows(prod, c)
    np.testing.assert_allclose(got[:, :32], want[:, :32], rtol=1e-6)
    raw = np.abs(ifg) / (a1 + np.float32(1e-12)) / (a2 + np.float32(1e-12))
    assert 0.1 < (raw > 1).mean() < 0.9  # both branches exercised
    np.testing.assert_allclose(got[:, 32:], want[:, 32:], rtol=2e-6, atol=1e-7)  # filled values included


def test_geometry_mirror_matches_oracle(cuda):
    rng = np.random.default_rng(1)
    llh = np.stack([rng.uniform(-80, 80, 500), rng.uniform(-180, 180, 500), rng.uniform(-400, 8000, 500)], axis=1)
    xyz = G.llh2xyz_vec(llh)
    np.testing.assert_allclose(xyz, og.llh2xyz(llh), rtol=0, atol=1e-7)
    back = G.xyz2llh_vec(xyz)
    want = og.xyz2llh(og.llh2xyz(llh))
    np.testing.assert_allclose(back[:, :2], want[..., :2], rtol=0, atol=1e-10)
    np.testing.assert_allclose(back[:, 2], want[..., 2], rtol=0, atol=1e-6)
    np.testing.assert_allclose(G.llh2xyz(llh[0]), og.llh2xyz(llh[0]), atol=1e-7)
    # line of sight from the middle state vector (s1proc/orbit.py:167-188)
    orb = synth.make_orbit(t_c=synth.ORBIT_T0 + 50.0)
    tt, xx, vv = orb
    sc = synth.make_radar_pair("tiny", seed=3)
    pts = np.stack([sc.lat.numpy().ravel()[::97], sc.lon.numpy().ravel()[::97], sc.hgt.numpy().ravel()[::97]], 1)
    los = G.orbitrangetime_vec(pts, tt, xx, vv)
    mid = len(tt) // 2
    _, dr, _ = og.orbitrangetime(tt, xx, vv, og.llh2xyz(pts), tt[mid], xx[mid], vv[mid])
    want_los = dr / np.linalg.norm(dr, axis=1, keepdims=True)
    assert np.abs(los - want_los).max() < 1e-9
    x, v = G.interp_orbit(tt, xx, vv, float(tt[mid]) + 1.3)
    xo, vo = og.intp_orbit(tt, xx, vv, np.float64(tt[mid] + 1.3))
    assert np.abs(x - xo).max() < 1e-6 and np.abs(v - vo).max() < 1e-8


@pytest.mark.parametrize("shape", [(70, 300), (1, 129)])
def test_los_grid_matches_oracle(cuda, shape):
    """s1proc/utils.py:240-292 (_los) on a DEM grid: float32 LOS vectors within
    a few ulps and look angles within 2e-5 degrees of the float64 oracle."""
    from types import SimpleNamespace
    sc = synth.make_pair("tiny", seed=7)
    tt, xx, vv = sc.ref[0].orbit
    orb = np.column_stack([tt, xx, vv])
    nlat, nlon = shape
    r = sc.rsc
    rsc = SimpleNamespace(latmax=r.latmax + 3 * r.dlat, lonmin=r.lonmin + 5 * r.dlon, dlat=r.dlat, dlon=r.dlon,
                          nlat=nlat, nlon=nlon)
    dem = np.random.default_rng(nlat * nlon).integers(-50, 3000, size=(nlat, nlon)).astype(np.int16)
    losvec, theta = G.los(orb, dem, rsc)
    want_los, want_theta = og.los_grid(orb, dem, rsc.latmax, rsc.lonmin, rsc.dlat, rsc.dlon, nlat, nlon)
    assert losvec.dtype == np.float32 and losvec.shape == (nlat * nlon, 3)
    assert theta.dtype == np.float32 and theta.shape == (nlat, nlon)
    assert np.abs(losvec - want_los).max() < 3e-7
    assert np.abs(theta - want_theta).max() < 2e-5
