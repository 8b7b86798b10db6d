"""The frame autotuner's cache on the GPU: the first autotune of a frame
times the candidates and writes its choice under this GPU and the frame's
shape class; a second chain of the same shape class takes the choice from
the cache without timing, and its products equal the first chain's."""
import pytest
import torch

from sentinel_gpu_processor_b200 import chain as C
from sentinel_gpu_processor_b200 import synth

pytestmark = pytest.mark.gpu


def test_autotune_cache_round_trip(cuda, tmp_path, monkeypatch):
    path = tmp_path / "tune.json"
    monkeypatch.setenv("S1B_TUNING_CACHE", str(path))
    sc = synth.make_frame(device=cuda, n_swaths=1, n_bursts=2, scale=0.12)

    def make():
        ch = C.BatchedFrameChain(sc.ref, sc.sec, sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=cuda,
                                 crossmul_fused=False, deramp_fused=False)
        for v, s in zip(ch.ref_views + ch.sec_views, sc.ref_slc + sc.sec_slc):
            v.copy_(s)
        return ch

    a = make()
    ta = a.autotune(sc.dem, reps=1)
    assert a.tuning_source == "timed"
    entries = C.load_tuning(str(path))
    assert list(entries.values()) == [ta]
    b = make()
    b.set_tuning(deramp_rows=8, deramp_ctas=1, geo_cols=256, geo_ctas=1)
    tb = b.autotune(sc.dem, reps=1)
    assert b.tuning_source == "cache" and tb == ta
    a.run(sc.dem)
    b.run(sc.dem)
    torch.cuda.synchronize()
    for ra, rb in zip(a.results(), b.results()):
        assert torch.equal(ra.ifg, rb.ifg) and torch.equal(ra.coh, rb.coh)
