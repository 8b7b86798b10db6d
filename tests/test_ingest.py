"""Measurement-TIFF ingest on the host (no GPU): the directory parser and
row reads of ``ingest.MeasurementTiff`` against a hand-assembled TIFF and
against rasters written in every layout the reader accepts (strips, tiles,
BigTIFF, big-endian, two int16 samples per pixel, zip members stored and
deflated).  The reference reads these files through GDAL
(s1proc/sentinel_scene.py:164-207); the values must come back exactly."""
import struct
import zipfile

import numpy as np
import pytest

from helpers import write_cint16_tiff
from sentinel_gpu_processor_b200.ingest import MeasurementTiff


def _raster(h, w, seed):
    rng = np.random.default_rng(seed)
    return rng.integers(-32768, 32768, size=(h, w, 2), dtype=np.int16)


def test_hand_assembled_tiff(tmp_path):
    # 3 samples x 2 lines, classic little-endian, one strip right after an
    # inline-only directory: CInt16 samples (re, im) = (10 r + c, -c)
    w, h = 3, 2
    ntag = 9
    data_off = 8 + 2 + 12 * ntag + 4
    ent = [(256, 3, 1, w), (257, 3, 1, h), (258, 3, 1, 32), (259, 3, 1, 1), (273, 4, 1, data_off),
           (277, 3, 1, 1), (278, 3, 1, h), (279, 4, 1, w * h * 4), (339, 3, 1, 5)]
    b = b"II" + struct.pack("<HI", 42, 8) + struct.pack("<H", ntag)
    for tag, typ, cnt, val in ent:
        b += struct.pack("<HHI", tag, typ, cnt) + (struct.pack("<HH", val, 0) if typ == 3 else struct.pack("<I", val))
    b += struct.pack("<I", 0)
    assert len(b) == data_off
    for r in range(h):
        for c in range(w):
            b += struct.pack("<hh", 10 * r + c, -c)
    p = tmp_path / "hand.tiff"
    p.write_bytes(b)
    with MeasurementTiff(str(p)) as t:
        assert (t.width, t.height) == (w, h)
        got = t.read_rows(0, 2)
    want = np.array([[[10 * r + c, -c] for c in range(w)] for r in range(h)], dtype=np.int16)
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("kw", [dict(rows_per_strip=1), dict(rows_per_strip=7), dict(),
                                dict(tile=(16, 16)), dict(tile=(32, 8)), dict(big=True, rows_per_strip=5),
                                dict(byteorder=">", rows_per_strip=4), dict(byteorder=">", tile=(16, 16), big=True),
                                dict(two_samples=True, rows_per_strip=3)])
def test_layouts_round_trip(tmp_path, kw):
    a = _raster(37, 45, 3)
    p = str(tmp_path / "m.tiff")
    write_cint16_tiff(p, a, **kw)
    with MeasurementTiff(p) as t:
        assert (t.width, t.height) == (45, 37)
        np.testing.assert_array_equal(t.read_rows(0, 37), a)
        np.testing.assert_array_equal(t.read_rows(5, 13), a[5:18])
        np.testing.assert_array_equal(t.read_rows(36, 1), a[36:])
        assert t.read_rows(10, 0).shape == (0, 45, 2)


def test_bursts_into_given_buffer(tmp_path):
    L, n, w = 6, 4, 20
    a = _raster(L * n, w, 5)
    p = str(tmp_path / "b.tiff")
    write_cint16_tiff(p, a, rows_per_strip=4)
    out = np.full((L, w, 2), 7, dtype=np.int16)
    with MeasurementTiff(p) as t:
        for k in range(n):
            assert t.read_burst(k, L, out) is out
            np.testing.assert_array_equal(out, a[k * L:(k + 1) * L])


@pytest.mark.parametrize("method", [zipfile.ZIP_STORED, zipfile.ZIP_DEFLATED])
def test_zip_member(tmp_path, method):
    a = _raster(30, 22, 9)
    p = str(tmp_path / "s1.tiff")
    write_cint16_tiff(p, a, rows_per_strip=1)
    z = str(tmp_path / "S1_SAFE.zip")
    with zipfile.ZipFile(z, "w", compression=method) as zf:
        zf.writestr("S1_SAFE/manifest.safe", "<xml/>")
        zf.write(p, "S1_SAFE/measurement/s1-iw1-slc-vv.tiff")
    with MeasurementTiff(z, "S1_SAFE/measurement/s1-iw1-slc-vv.tiff") as t:
        np.testing.assert_array_equal(t.read_rows(0, 30), a)
        np.testing.assert_array_equal(t.read_rows(11, 9), a[11:20])
        np.testing.assert_array_equal(t.read_rows(2, 3), a[2:5])  # backwards after a later read


def test_rejections(tmp_path):
    a = _raster(8, 8, 1)
    p = str(tmp_path / "c.tiff")
    write_cint16_tiff(p, a, compression=8)
    with pytest.raises(ValueError, match="compressed"):
        MeasurementTiff(p)
    bad = tmp_path / "not.tiff"
    bad.write_bytes(b"GIF89a" + bytes(20))
    with pytest.raises(ValueError, match="not a TIFF"):
        MeasurementTiff(str(bad))
    p2 = str(tmp_path / "ok.tiff")
    write_cint16_tiff(p2, a)
    with MeasurementTiff(p2) as t:
        with pytest.raises(ValueError, match="outside"):
            t.read_rows(5, 4)
        with pytest.raises(ValueError, match="out must be"):
            t.read_rows(0, 2, np.empty((2, 8, 2), dtype=np.int32))
