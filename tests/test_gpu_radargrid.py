"""Radar-grid coregistration on the GPU (geo2rdr offsets from lat/lon/height
rasters, TOPS-aware 8-tap sinc / bilinear resampling, 5x5 box coherence)
against the float64 oracle (oracle/radargrid.py).

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
def scene():
    return synth.make_radar_pair("tiny", seed=11)


def _plan(acq):
    return P.burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, acq.bursts[0], None)


def test_offsets_match_oracle(cuda, scene):
    pl = _plan(scene.sec)
    az, rg = kernels.geo2rdr_offsets(pl, scene.lat.to(cuda), scene.lon.to(cuda), scene.hgt.to(cuda))
    oaz, org, _, _ = orr.offsets(scene.lat.numpy(), scene.lon.numpy(), scene.hgt.numpy(), oracle_radar(scene.sec.radar),
                                 scene.sec.orbit, scene.sec.bursts[0].azimuth_time)
    assert np.abs(az.cpu().numpy() - oaz).max() < 1e-4
    assert np.abs(rg.cpu().numpy() - org).max() < 1e-4
    # the reference grid geocoded on its own orbit is the identity
    pr = _plan(scene.ref)
    az0, rg0 = kernels.geo2rdr_offsets(pr, scene.lat.to(cuda), scene.lon.to(cuda), scene.hgt.to(cuda))
    assert az0.abs().max() < 1e-4 and rg0.abs().max() < 1e-4


@pytest.mark.parametrize("interp", ["sinc8", "bilinear"])
def test_resample_matches_oracle(cuda, scene, interp):
    pl = _plan(scene.sec)
    az, rg = kernels.geo2rdr_offsets(pl, scene.lat.to(cuda), scene.lon.to(cuda), scene.hgt.to(cuda))
    got = kernels.resample(pl, scene.sec_slc.to(cuda), az, rg, interp=interp).cpu().numpy()
    L, S = az.shape
    A = np.arange(L)[:, None] + az.cpu().numpy().astype(np.float64)
    R = np.arange(S)[None, :] + rg.cpu().numpy().astype(np.float64)
    co = og2.burst_coefficients(oracle_radar(scene.sec.radar), scene.sec.orbit, scene.sec.fm, scene.sec.dc,
                                oracle_burst(scene.sec.bursts[0]))
    want, ok = orr.resample(scene.sec_slc.numpy(), oracle_radar(scene.sec.radar), co, A, R, interp)
    assert ok.mean() > 0.8
    assert np.array_equal(np.abs(got) > 0, np.abs(want) > 0)
    assert rel_err(got, want) < 2e-5
    assert phase_rms(got, want, ok) < 1e-3


def _oracle_resample(acq, sec_slc, az, rg, interp="sinc8"):
    L, S = az.shape
    A = np.arange(L)[:, None] + az.cpu().numpy().astype(np.float64)
    R = np.arange(S)[None, :] + rg.cpu().numpy().astype(np.float64)
    co = og2.burst_coefficients(oracle_radar(acq.radar), acq.orbit, acq.fm, acq.dc, oracle_burst(acq.bursts[0]))
    return orr.resample(sec_slc.cpu().numpy(), oracle_radar(acq.radar), co, A, R, interp)


@pytest.fixture(scope="module")
def scene_c0(cuda):
    return synth.make_radar_pair("c0", seed=13, device=cuda)


def test_resample_pipeline_matches_oracle(cuda, scene_c0):
    """512 x 2048: 1024 tiles, several per persistent CTA, so the TMA stages
    (three offset stages, two window stages) rotate; status stays 0."""
    sc = scene_c0
    pl = _plan(sc.sec)
    az, rg = kernels.geo2rdr_offsets(pl, sc.lat, sc.lon, sc.hgt)
    status = torch.full((1,), 7, dtype=torch.int32, device=cuda)
    got = kernels.resample(pl, sc.sec_slc, az, rg, status=status).cpu().numpy()
    assert status.item() == 0
    want, ok = _oracle_resample(sc.sec, sc.sec_slc, az, rg)
    assert ok.mean() > 0.9
    assert np.array_equal(np.abs(got) > 0, np.abs(want) > 0)
    assert rel_err(got, want) < 2e-5
    assert phase_rms(got, want, ok) < 1e-3


@pytest.mark.parametrize("cols", [317, 318])
def test_resample_plain_load_path(cuda, scene, cols):
    """Widths whose offset rows are not a multiple of 16 bytes (no tensor map)
    take the plain-load kernel; results agree with the oracle and with the
    TMA kernel on the columns both cover."""
    pl = _plan(scene.sec)
    az, rg = kernels.geo2rdr_offsets(pl, scene.lat.to(cuda), scene.lon.to(cuda), scene.hgt.to(cuda))
    sec = scene.sec_slc.to(cuda)
    azc, rgc = az[:, :cols].contiguous(), rg[:, :cols].contiguous()
    got = kernels.resample(pl, sec, azc, rgc).cpu().numpy()
    want, ok = _oracle_resample(scene.sec, sec, azc, rgc)
    assert rel_err(got, want) < 2e-5
    full = kernels.resample(pl, sec, az, rg).cpu().numpy()[:, :cols]
    assert rel_err(got, full) < 1e-5


def test_resample_with_large_offsets_uses_direct_path(cuda, scene):
    """Offsets that vary too much inside a tile for the staged window take the
    per-tap path; results must not change."""
    pl = _plan(scene.sec)
    L, S = scene.lat.shape
    rng = np.random.default_rng(1)
    az = torch.from_numpy(rng.uniform(-20, 20, (L, S)).astype(np.float32)).to(cuda)
    rg = torch.from_numpy(rng.uniform(-30, 30, (L, S)).astype(np.float32)).to(cuda)
    got = kernels.resample(pl, scene.sec_slc.to(cuda), az, rg).cpu().numpy()
    co = og2.burst_coefficients(oracle_radar(scene.sec.radar), scene.sec.orbit, scene.sec.fm, scene.sec.dc,
                                oracle_burst(scene.sec.bursts[0]))
    A = np.arange(L)[:, None] + az.cpu().numpy().astype(np.float64)
    R = np.arange(S)[None, :] + rg.cpu().numpy().astype(np.float64)
    want, ok = orr.resample(scene.sec_slc.numpy(), oracle_radar(scene.sec.radar), co, A, R, "sinc8")
    assert rel_err(got, want) < 2e-5


@pytest.mark.parametrize("shape,win", [((96, 320), 5), ((70, 257), 5), ((33, 130), 3), ((40, 128), 9),
                                       ((50, 200), 1), ((66, 136), 7), ((97, 390), 9)])
def test_box_coherence_matches_oracle(cuda, shape, win):
    rng = np.random.default_rng(shape[0] + win)
    a = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    n = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    b = (0.8 * a * np.exp(1j * 0.3) + 0.6 * n).astype(np.complex64)
    # a zero patch: windows inside it have zero power and coherence 0
    a[10:30, 40:70] = 0
    got = kernels.box_coherence(torch.from_numpy(a).to(cuda), torch.from_numpy(b).to(cuda), win).cpu().numpy()
    want = orr.box_coherence(a, b, win)
    assert np.abs(got - want).max() < 1e-4
    h = win // 2
    assert (got[10 + h:30 - h, 40 + h:70 - h] == 0).all()


def test_resampled_pair_is_coherent(cuda):
    """End to end on a consistent synthetic pair: after resampling, the 5x5
    coherence is high where the secondary was simulated coherent (0.9)."""
    sc = synth.make_radar_pair("tiny", seed=12, coherence=0.9)
    pl = _plan(sc.sec)
    az, rg = kernels.geo2rdr_offsets(pl, sc.lat.to(cuda), sc.lon.to(cuda), sc.hgt.to(cuda))
    res = kernels.resample(pl, sc.sec_slc.to(cuda), az, rg)
    # deramp the reference the same way so both carry no TOPS phase difference
    ref = sc.ref_slc.to(cuda)
    g = kernels.box_coherence(ref, res, 5).cpu().numpy()[8:-8, 8:-8]
    assert np.median(g) > 0.7


def test_radar_chain_graph_replay_matches_eager(cuda):
    """The radar-grid chain captured in a CUDA graph reproduces the eager
    step bit for bit, and no tile lost a staging copy."""
    from sentinel_gpu_processor_b200.chain import RadarChain
    sc = synth.make_radar_pair("small", seed=21, device=cuda)
    L, S = sc.ref_slc.shape
    ch = RadarChain(sc.ref, sc.sec, L, S, sc.rowlook, sc.collook, sc.alpha, device=cuda)
    ins = (sc.ref_slc, sc.sec_slc, sc.lat, sc.lon, sc.hgt)
    eager = {k: v.clone() for k, v in ch.run(*ins).items()}
    ch.capture(*ins)
    for k in ("ifg", "coh_full", "filt"):
        ch.outs[k].zero_()
    out = ch.replay()
    torch.cuda.synchronize()
    assert out is not None and ch.staging_ok()
    for k in ("ifg", "coh_full", "filt"):
        assert torch.equal(out[k], eager[k]), k
    assert float(out["coh_full"][8:-8, 8:-8].median()) > 0.3
