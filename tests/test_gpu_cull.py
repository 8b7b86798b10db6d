"""Culling of the geocoding blocks that lie outside a burst's valid lines:
the products with culling equal those without it bit for bit -- single
bursts of the synthetic scenes, DEMs whose heights reach both ends of the
int16 range (which move a pixel's azimuth line the most), and a batched
frame -- so culling drops only pixels that are zero in the reference's
output (geo2rdr.cu:208-209)."""
import numpy as np
import pytest
import torch

from sentinel_gpu_processor_b200 import kernels, plan as P, synth
from sentinel_gpu_processor_b200.chain import BatchedFrameChain

pytestmark = pytest.mark.gpu


@pytest.fixture
def culling(cuda):
    """Sets culling for the test; restores the default (on) afterwards."""
    yield kernels.set_geocode_culling
    kernels.set_geocode_culling(True)


def _geocode_both(culling, pl, dem, deramped):
    outs = []
    for on in (True, False):
        culling(on)
        out, rows = kernels.geo2rdr(pl, dem, deramped)
        torch.cuda.synchronize()
        outs.append((out.clone(), rows.clone()))
    return outs


def _equal(a, b):
    assert torch.equal(torch.view_as_real(a[0]), torch.view_as_real(b[0]))
    assert torch.equal(a[1], b[1])


@pytest.mark.parametrize("cfg,seed", [("tiny", 41), ("small", 42)])
def test_culling_gives_identical_bursts(cuda, culling, cfg, seed):
    sc = synth.make_pair(cfg, seed=seed)
    dem = sc.dem.to(cuda)
    n_zero = 0
    for acq, slc in ((sc.ref[0], sc.ref_slc[0]), (sc.sec[0], sc.sec_slc[0])):
        pl = P.burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, acq.bursts[0], sc.rsc)
        der = kernels.deramp(pl, slc.to(cuda))
        a, b = _geocode_both(culling, pl, dem, der)
        _equal(a, b)
        n_zero += int((a[0] == 0).sum())
    assert n_zero > 0  # the windows hold pixels outside the bursts


def test_culling_with_extreme_heights(cuda, culling):
    """Heights of -32768 and 32767 m scattered over the DEM and in whole
    blocks: a culled block must stay outside the valid lines at any height."""
    sc = synth.make_pair("small", seed=43)
    acq = sc.ref[0]
    pl = P.burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, acq.bursts[0], sc.rsc)
    der = kernels.deramp(pl, sc.ref_slc[0].to(cuda))
    rng = np.random.default_rng(5)
    dem = sc.dem.numpy().copy()
    m = rng.uniform(size=dem.shape)
    dem[m < 0.05] = 32767
    dem[m > 0.95] = -32768
    dem[:64, :] = 32767
    dem[-64:, :] = -32768
    dem[:, :64] = -32768
    a, b = _geocode_both(culling, pl, torch.from_numpy(dem).to(cuda), der)
    _equal(a, b)
    assert int((a[0] != 0).sum()) > 0


def test_culling_gives_identical_frames(cuda, culling):
    f = synth.make_frame(seed=9, device=cuda, n_swaths=2, n_bursts=2, scale=0.12)
    outs = []
    for on in (True, False):
        culling(on)
        bc = BatchedFrameChain(f.ref, f.sec, f.rsc, f.rowlook, f.collook, f.alpha, device=cuda)
        bc.load(f.ref_slc, f.sec_slc)
        bc.run(f.dem)
        torch.cuda.synchronize()
        outs.append([None if r is None else [list(r.header), tuple(r.box)]
                     + [getattr(r, k).clone() for k in ("ifg", "amp1", "amp2", "coh", "filt")]
                     for r in bc.results()])
    assert any(r is not None for r in outs[0])
    for a, b in zip(*outs):
        assert (a is None) == (b is None)
        if a is not None:
            assert a[:2] == b[:2]
            for x, y in zip(a[2:], b[2:]):
                assert torch.equal(torch.view_as_real(x) if x.is_complex() else x,
                                   torch.view_as_real(y) if y.is_complex() else y)
