"""s1proc file formats round trip (CPU)."""
import numpy as np

from sentinel_gpu_processor_b200 import formats


def test_raster_roundtrip(tmp_path):
    h = formats.make_header(100, 200, 5, 7, 25, 17)
    d = (np.arange(200) + 1j * np.arange(200)).astype(np.complex64).reshape(10, 20)
    f = tmp_path / "a.gslc"
    formats.write_raster(f, h, d)
    h2, d2 = formats.read_raster(f)
    np.testing.assert_array_equal(h, h2)
    np.testing.assert_array_equal(d, d2)
    assert f.stat().st_size == 64 * 4 + 200 * 8


def test_truncated_raster_raises(tmp_path):
    h = formats.make_header(100, 200, 0, 0, 10, 10)
    f = tmp_path / "t.gslc"
    formats.write_raster(f, h, np.zeros(50, np.complex64))
    try:
        formats.read_raster(f)
    except IOError:
        pass
    else:
        raise AssertionError("truncated raster accepted")


def test_rsc_roundtrip_and_take_look(tmp_path):
    r = formats.rsc_roundtrip(formats.Rsc(1000, 2000, 36.5, 13.25, -1 / 7200, 1 / 7200))
    f = tmp_path / "d.rsc"
    formats.write_rsc(f, r)
    assert formats.read_rsc(f) == r
    lk = r.take_look(4, 20)
    assert (lk.nlat, lk.nlon) == (250, 100)
    assert abs(lk.latmax - (r.latmax + r.dlat * 1.5)) < 1e-15
    assert abs(lk.dlon - 20 * r.dlon) < 1e-18


def test_orbit_poly_db_roundtrip(tmp_path):
    tt = np.array([1.0, 11.0, 21.0, 31.0])
    xx = np.arange(12.0).reshape(4, 3) * 1e6 + 0.123456789
    vv = np.arange(12.0).reshape(4, 3) * 1.5
    f = tmp_path / "o.txt"
    formats.write_orbit_ascii(f, tt, xx, vv)
    t2, x2, v2 = formats.read_orbit_ascii(f)
    np.testing.assert_array_equal(tt, t2)
    np.testing.assert_array_equal(xx, x2)
    np.testing.assert_array_equal(vv, v2)
    tab = np.array([[1.5, 0.005, 1252.7, 3.2e4, 0.0], [4.5, 0.005, 1253.7, 3.3e4, 1e6]])
    fp = tmp_path / "fm.txt"
    formats.write_poly(fp, tab)
    np.testing.assert_array_equal(formats.read_poly(fp), tab)
    db = tmp_path / "p.db"
    formats.write_db(db, {"prf": 486.486, "linesPerBurst": 1500, "demfile": "/x/y.dem"})
    d = formats.read_db(db)
    assert float(d["prf"]) == 486.486 and int(d["linesPerBurst"]) == 1500 and d["demfile"] == "/x/y.dem"
