"""Host planner of libs1b (orbit polynomials, TOPS coefficients, footprint,
DEM window, crossmul box) against the float64 oracle.  CPU only."""
import numpy as np
import pytest

from helpers import oracle_burst, oracle_radar, oracle_rsc
from oracle import crossmul as ox
from oracle import geo2rdr as og2
from oracle import geometry as og
from sentinel_gpu_processor_b200 import formats, plan as P, synth


@pytest.fixture(scope="module", params=[("tiny", 1), ("small", 2), ("c0", 3)])
def scene(request):
    cfg, seed = request.param
    return synth.make_pair(cfg, seed=seed)


def test_orbit_polynomial_equals_hermite(scene):
    tt, xx, vv = scene.ref[0].orbit
    poly = P.orbit_poly(tt, xx, vv)
    t = np.linspace(tt[0] - 4.0, tt[-1] + 4.0, 3001)
    x1, v1 = P.orbit_eval(poly, t)
    x2, v2 = og.intp_orbit(tt, xx, vv, t)
    assert np.abs(x1 - x2).max() < 1e-6  # metres; observed ~1e-8
    assert np.abs(v1 - v2).max() < 1e-8


def test_burst_plan_matches_oracle(scene):
    for acq in (scene.ref[0], scene.sec[0]):
        pl = P.burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, acq.bursts[0], scene.rsc)
        r = oracle_radar(acq.radar)
        b = oracle_burst(acq.bursts[0])
        co = og2.burst_coefficients(r, acq.orbit, acq.fm, acq.dc, b)
        assert abs(pl.ks - co.ks) < 1e-9 * abs(co.ks)
        np.testing.assert_allclose(list(pl.fm), co.fm, rtol=1e-14)
        np.testing.assert_allclose(list(pl.dc), co.dc, rtol=1e-14)
        assert abs(pl.etac0 - co.etac0) < 1e-15
        box = og2.burst_latlon_box(r, acq.orbit, b)
        np.testing.assert_allclose(list(pl.latlon_box), box, rtol=0, atol=1e-9)
        w = og2.dem_window(box, oracle_rsc(scene.rsc))
        assert pl.window == (w.left, w.top, w.right, w.bottom)
        assert pl.nrow > 0 and pl.ncol > 0


def test_bounds_many_cases():
    tt, xx, vv = synth.make_orbit()
    poly = P.orbit_poly(tt, xx, vv)
    rng = np.random.default_rng(3)
    for _ in range(20):
        t0 = rng.uniform(tt[1], tt[-3])
        t1 = t0 + rng.uniform(0.5, 3.5)
        r0 = rng.uniform(7.9e5, 9.0e5)
        r1 = r0 + rng.uniform(1e4, 6e4)
        h0, h1 = -100.0, rng.uniform(500, 9000)
        got = P.bounds(poly, t0, t1, r0, r1, h0, h1)
        want = og.bounds(t0, t1, r0, r1, h0, h1, tt, xx, vv)
        np.testing.assert_allclose(got, want, rtol=0, atol=1e-9)


def test_crossmul_box_matches_oracle():
    rng = np.random.default_rng(4)
    for _ in range(300):
        rl, cl = int(rng.integers(1, 6)), int(rng.integers(1, 25))
        h = []
        for _k in range(2):
            l0 = int(rng.integers(0, 200))
            t0 = int(rng.integers(0, 200))
            h.append(formats.make_header(500, 800, l0, t0, l0 + int(rng.integers(1, 300)),
                                         t0 + int(rng.integers(1, 300))))
        box, hdr = P.crossmul_box(h[0], h[1], rl, cl)
        want = ox.intersection_box(h[0], h[1], rl, cl)
        if want is None:
            assert box is None
        else:
            assert tuple(box) == tuple(want)
            np.testing.assert_array_equal(hdr, ox.ifg_header(h[0], want, rl, cl)[:6])
        ubox, _ = P.crossmul_box(h[0], h[1], rl, cl, use_union=True)
        uwant = ox.union_box(h[0], h[1], rl, cl)
        assert (ubox is None) == (uwant is None)
        if uwant is not None:
            assert tuple(ubox) == tuple(uwant)


def test_plan_rejects_bad_input():
    from sentinel_gpu_processor_b200 import _lib
    sc = synth.make_pair("tiny", seed=9)
    acq = sc.ref[0]
    tt, xx, vv = acq.orbit
    with pytest.raises(_lib.S1BError):
        P.burst_plan(acq.radar, (tt[:3], xx[:3], vv[:3]), acq.fm, acq.dc, acq.bursts[0], sc.rsc)
    big = (np.arange(70) * 10.0, np.zeros((70, 3)), np.ones((70, 3)))
    with pytest.raises(_lib.S1BError):
        P.orbit_poly(*big)
