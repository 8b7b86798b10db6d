"""The bounded staging waits of the TMA resampler, made to run out.

Every shared-memory staging wait of resample_tma_kernel is bounded.  A wait
that gives up sets the call's status word, lets the block's copies in flight
land (a second bounded wait) and ends the block, so the context stays
usable.  The test hook s1b_set_staging_poll_limit(0) makes every wait give up
at once (no fault, no hang: nothing else changes); the status must read 1,
and with the default limit restored the next call must give status 0 and
the result of a run that never had the limit changed."""
import pytest
import torch

from sentinel_gpu_processor_b200 import _lib, kernels, plan as P, synth

pytestmark = pytest.mark.gpu


def test_resampler_wait_expiry_sets_status_and_context_survives(cuda):
    sc = synth.make_radar_pair("small", seed=31, device=cuda)
    pl = P.burst_plan(sc.sec.radar, sc.sec.orbit, sc.sec.fm, sc.sec.dc, sc.sec.bursts[0], None)
    az, rg = kernels.geo2rdr_offsets(pl, sc.lat, sc.lon, sc.hgt)
    status = torch.zeros(1, dtype=torch.int32, device=cuda)
    want = kernels.resample(pl, sc.sec_slc, az, rg, status=status)
    torch.cuda.synchronize()
    assert status.item() == 0
    lib = _lib.load()
    prev = lib.s1b_set_staging_poll_limit(0)
    try:
        status.fill_(0)
        kernels.resample(pl, sc.sec_slc, az, rg, status=status)
        torch.cuda.synchronize()
        assert status.item() == 1
    finally:
        lib.s1b_set_staging_poll_limit(prev)
    assert prev == 1 << 22
    status.fill_(7)
    again = kernels.resample(pl, sc.sec_slc, az, rg, status=status)
    torch.cuda.synchronize()
    assert status.item() == 0
    assert torch.equal(again, want)
