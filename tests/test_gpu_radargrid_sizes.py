"""The radar-grid chain at the workload size C1 (one 1500 x 21000 burst pair
with float64 lat/lon/height rasters): geo2rdr offsets on the secondary
orbit, the TOPS-aware 8-tap sinc resampler and the 5 x 5 box coherence,
against the float64 oracle (oracle/radargrid.py) on rows spread over the
whole burst (the oracle is too slow for all 31.5 M pixels; the kernels run
on the whole burst, so every tile schedule, TMA stage and CTA of the
full-size launch is exercised).  The 512 x 2048 case (C0) is covered in
test_gpu_radargrid.py.

Tolerances (north star): offsets <= 1e-4 px, RMS wrapped phase <= 1e-3 rad,
coherence |delta| <= 1e-4.
"""
import numpy as np
import pytest
import torch

from helpers import oracle_burst, oracle_radar, phase_rms, rel_err
from oracle import geo2rdr as og2
from oracle import radargrid as orr
from sentinel_gpu_processor_b200 import kernels, plan as P, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1(cuda):
    sc = synth.make_radar_pair("c1", seed=20261203 + 1200, device=cuda)
    pl = P.burst_plan(sc.sec.radar, sc.sec.orbit, sc.sec.fm, sc.sec.dc, sc.sec.bursts[0], None)
    az, rg = kernels.geo2rdr_offsets(pl, sc.lat, sc.lon, sc.hgt)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    res = kernels.resample(pl, sc.sec_slc, az, rg, status=status)
    coh = kernels.box_coherence(sc.ref_slc, res, 5, status=status)
    torch.cuda.synchronize()
    assert status.item() == 0
    L, S = az.shape
    rows = np.linspace(40, L - 41, 7).round().astype(np.int64)
    return dict(sc=sc, pl=pl, az=az, rg=rg, res=res, coh=coh, rows=rows, L=L, S=S)


def test_c1_offsets_match_oracle(c1):
    sc, rows = c1["sc"], c1["rows"]
    lat, lon, hgt = (t[rows].cpu().numpy() for t in (sc.lat, sc.lon, sc.hgt))
    _, _, oaz, org = orr.offsets(lat, lon, hgt, oracle_radar(sc.sec.radar), sc.sec.orbit, sc.sec.bursts[0].azimuth_time)
    gaz = rows[:, None] + c1["az"][rows].cpu().numpy().astype(np.float64)
    grg = np.arange(c1["S"])[None, :] + c1["rg"][rows].cpu().numpy().astype(np.float64)
    assert np.abs(gaz - oaz).max() < 1e-4
    assert np.abs(grg - org).max() < 1e-4


def test_c1_resample_matches_oracle(c1):
    sc, rows = c1["sc"], c1["rows"]
    A = rows[:, None] + c1["az"][rows].cpu().numpy().astype(np.float64)
    R = np.arange(c1["S"])[None, :] + c1["rg"][rows].cpu().numpy().astype(np.float64)
    co = og2.burst_coefficients(oracle_radar(sc.sec.radar), sc.sec.orbit, sc.sec.fm, sc.sec.dc,
                                oracle_burst(sc.sec.bursts[0]))
    want, ok = orr.resample(sc.sec_slc.cpu().numpy(), oracle_radar(sc.sec.radar), co, A, R, "sinc8")
    got = c1["res"][rows].cpu().numpy()
    assert ok.mean() > 0.9
    assert np.array_equal(np.abs(got) > 0, np.abs(want) > 0)
    assert rel_err(got, want) < 2e-5
    assert phase_rms(got, want, ok) < 1e-3


def test_c1_box_coherence_matches_oracle(c1):
    sc, rows = c1["sc"], c1["rows"]
    for r in rows:
        a = sc.ref_slc[r - 2:r + 3].cpu().numpy()
        b = c1["res"][r - 2:r + 3].cpu().numpy()
        want = orr.box_coherence(a, b, 5)[2]  # the middle row has its whole 5-row window
        got = c1["coh"][r].cpu().numpy()
        assert np.abs(got - want).max() < 1e-4
    assert float(c1["coh"][100:-100, 100:-100].median()) > 0.3
