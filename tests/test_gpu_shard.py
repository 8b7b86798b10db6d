"""A frame split over two ranks (``shard.frame_shard``) gives, pair for pair,
the same products as the whole frame: the two shards are run one after the
other on this GPU, each as its own ``BatchedFrameChain`` (no rank waits on
another)."""
import pytest
import torch

from sentinel_gpu_processor_b200 import shard, synth
from sentinel_gpu_processor_b200.chain import BatchedFrameChain

pytestmark = pytest.mark.gpu


def _run(refs, secs, ref_slc, sec_slc, sc, cuda):
    ch = BatchedFrameChain(refs, secs, sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=cuda)
    for v, s in zip(ch.ref_views + ch.sec_views, list(ref_slc) + list(sec_slc)):
        v.copy_(s)
    ch.run(sc.dem)
    torch.cuda.synchronize()
    return ch.results()


def test_shards_reproduce_the_whole_frame(cuda):
    sc = synth.make_frame(device=cuda, n_swaths=1, n_bursts=5, scale=0.12)
    whole = _run(sc.ref, sc.sec, sc.ref_slc, sc.sec_slc, sc, cuda)
    seen = []
    for rank in range(2):
        idx, refs, secs = shard.frame_shard(sc.ref, sc.sec, rank, 2)
        part = _run(refs, secs, [sc.ref_slc[k] for k in idx], [sc.sec_slc[k] for k in idx], sc, cuda)
        for k, r in zip(idx, part):
            w = whole[k]
            assert (r is None) == (w is None)
            if r is not None:
                assert torch.equal(r.ifg, w.ifg) and torch.equal(r.coh, w.coh) and torch.equal(r.filt, w.filt)
        seen += idx
    assert sorted(seen) == list(range(len(sc.ref)))
