"""Burst geometry prep on the GPU (s1b_burst_geometry): the footprint at
hmin..hmax, the DEM window and the TOPS centre terms (ks, interpolated
FM-rate / Doppler polynomials, etac0) of every burst of a full IW frame (54
bursts) and of a time-series stack's reference and secondary dates in one
launch, against the host planner (s1b_burst_plan) and the float64 oracle
(bounds restated from csrc/src/bounds.cu, pinned to the reference's own
compiled code in test_oracle_pins.py)."""
import numpy as np
import pytest

from helpers import oracle_burst, oracle_radar
from oracle import geo2rdr as og2
from sentinel_gpu_processor_b200 import plan as P, synth

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scene", ["frame", "stack"])
def test_device_geometry_matches_host_planner_and_oracle(cuda, scene):
    if scene == "frame":
        sc = synth.make_frame(slc_pairs=0, with_dem=False)
        acqs, rsc = sc.ref + sc.sec, sc.rsc
    else:
        st = synth.make_stack(with_dem=False, n_sec=6)
        acqs, rsc = st.ref + [a for d in st.sec for a in d], st.rsc
    got = P.burst_geometry_device(acqs, rsc, cuda)
    assert len(got) == len(acqs)
    for g, a in zip(got, acqs):
        assert g.status == 0
        pl = P.burst_plan(a.radar, a.orbit, a.fm, a.dc, a.bursts[0], rsc)
        np.testing.assert_allclose(list(g.latlon_box), list(pl.latlon_box), rtol=0, atol=1e-11)
        assert list(g.win) == [pl.win_left, pl.win_top, pl.win_right, pl.win_bottom]
        np.testing.assert_allclose([g.ks, g.etac0, *g.fm, *g.dc], [pl.ks, pl.etac0, *pl.fm, *pl.dc], rtol=1e-13)
        box = og2.burst_latlon_box(oracle_radar(a.radar), a.orbit, oracle_burst(a.bursts[0]))
        np.testing.assert_allclose(list(g.latlon_box), box, rtol=0, atol=1e-9)
        co = og2.burst_coefficients(oracle_radar(a.radar), a.orbit, a.fm, a.dc, oracle_burst(a.bursts[0]))
        np.testing.assert_allclose([g.ks, *g.fm, *g.dc, g.etac0], [co.ks, *co.fm, *co.dc, co.etac0], rtol=1e-9)


def test_device_geometry_flags_bad_records(cuda):
    sc = synth.make_pair("tiny", seed=3)
    acq = sc.ref[0]
    bad = type(acq)(radar=synth.make_radar(1, 320), orbit=acq.orbit, fm=acq.fm, dc=acq.dc, bursts=acq.bursts)
    g = P.burst_geometry_device([acq, bad], sc.rsc, cuda)
    assert g[0].status == 0 and g[1].status == 1
