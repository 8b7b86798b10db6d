"""The time-series stack's synthetic dates see one scene: every secondary
date's SLC holds the reference's band-limited speckle at its own sample
positions of the same ground points (``synth.locked_to_reference``), so the
geocoded interferograms of the batched frame path are coherent at about the
date's simulated coherence, and less so for later dates."""
import pytest
import torch

from sentinel_gpu_processor_b200 import synth
from sentinel_gpu_processor_b200.chain import BatchedFrameChain

pytestmark = pytest.mark.gpu


def test_stack_pairs_coherent_at_simulated_coherence(cuda):
    st = synth.make_stack(device=cuda, n_sec=3, n_bursts=2, lines=600, samples=4000)
    nb = st.n_bursts
    acqs = list(st.ref) + [st.sec[d][b] for d in range(3) for b in range(nb)]
    pairs = [(b, nb + d * nb + b) for d in range(3) for b in range(nb)]
    ch = BatchedFrameChain(acqs, None, st.rsc, st.rowlook, st.collook, st.alpha, device=cuda, pairs=pairs)
    for b in range(nb):
        ch.views[b].copy_(synth.stack_slc(st, -1, b, cuda))
    for d in range(3):
        for b in range(nb):
            ch.views[nb + d * nb + b].copy_(synth.stack_slc(st, d, b, cuda))
    ch.capture(st.dem)
    ch.replay()
    torch.cuda.synchronize()
    med = {}
    for k, r in enumerate(ch.results()):
        c = r.coh.float()
        med.setdefault(k // nb, []).append(float(c[c > 0].median()))
    for d in range(3):
        g = st.coherence[d]
        for m in med[d]:
            # interpolation by the geocoding's bilinear gathers costs ~10 %
            assert 0.75 * g < m < 1.05 * g, (d, g, med[d])
    assert min(med[0]) > max(med[2])


def test_frame_pairs_ground_locked_coherent(cuda):
    """The frame's pairs made by ``synth.ground_lock_pairs`` (the bench's
    headline workload) are coherent at about their simulated coherence."""
    sc = synth.make_frame(device=cuda, n_swaths=1, n_bursts=3, scale=0.25, slc_pairs=0)
    synth.ground_lock_pairs(sc, range(len(sc.ref)))
    ch = BatchedFrameChain(sc.ref, sc.sec, sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=cuda)
    for v, s in zip(ch.ref_views + ch.sec_views, sc.ref_slc + sc.sec_slc):
        v.copy_(s)
    ch.capture(sc.dem)
    ch.replay()
    torch.cuda.synchronize()
    for k, r in enumerate(ch.results()):
        c = r.coh.float()
        m = float(c[c > 0].mean())
        g = sc.extra["coherence"][k]
        assert 0.8 * g < m < 1.1 * g, (k, g, m)
