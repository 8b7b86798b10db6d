"""Crossmul + multilook + coherence parity on the GPU against the oracle
(oracle/crossmul.py, oracle/coherence.py).

Tolerances: interferogram relative error <= 1e-5 of its peak (float32
summation order differs), RMS wrapped phase <= 1e-3 rad, coherence
|delta| <= 1e-4 (north star).
"""
import numpy as np
import pytest
import torch

from helpers import phase_rms, rel_err
from oracle import coherence as oc
from oracle import crossmul as ox
from sentinel_gpu_processor_b200 import formats, interfere, kernels

pytestmark = pytest.mark.gpu


def _pair(rng, h1, h2, corr=0.8):
    n1 = (h1[5] - h1[3], h1[4] - h1[2])
    n2 = (h2[5] - h2[3], h2[4] - h2[2])
    d1 = (rng.standard_normal(n1) + 1j * rng.standard_normal(n1)).astype(np.complex64)
    d2 = (rng.standard_normal(n2) + 1j * rng.standard_normal(n2)).astype(np.complex64)
    # correlate the overlap so coherence is non-trivial
    l, t = max(h1[2], h2[2]), max(h1[3], h2[3])
    r, b = min(h1[4], h2[4]), min(h1[5], h2[5])
    if l < r and t < b:
        a = d1[t - h1[3]:b - h1[3], l - h1[2]:r - h1[2]]
        ph = np.exp(1j * np.linspace(0, 6, a.shape[1]))[None, :]
        d2[t - h2[3]:b - h2[3], l - h2[2]:r - h2[2]] = (corr * a * ph + np.sqrt(1 - corr ** 2) *
                                                          d2[t - h2[3]:b - h2[3], l - h2[2]:r - h2[2]])
    return d1, d2.astype(np.complex64)


CASES = [
    # (h1, h2, rowlook, collook)
    (formats.make_header(400, 900, 10, 7, 610, 203), formats.make_header(400, 900, 23, 3, 640, 190), 4, 20),
    (formats.make_header(400, 900, 0, 0, 333, 101), formats.make_header(400, 900, 5, 2, 333, 101), 2, 8),
    (formats.make_header(100, 100, 3, 4, 77, 61), formats.make_header(100, 100, 1, 1, 70, 66), 1, 1),
    (formats.make_header(100, 3000, 0, 0, 2100, 40), formats.make_header(100, 3000, 7, 0, 2100, 40), 3, 700),
]


@pytest.mark.parametrize("h1,h2,rl,cl", CASES)
def test_crossmul_looks_matches_oracle(cuda, h1, h2, rl, cl):
    rng = np.random.default_rng(rl * 1000 + cl)
    d1, d2 = _pair(rng, h1, h2)
    r = interfere.crossmul_pair(h1, torch.from_numpy(d1).to(cuda), h2, torch.from_numpy(d2).to(cuda), rl, cl)
    want = ox.crossmul_pair(h1, d1, h2, d2, rl, cl)
    assert r is not None and want is not None
    np.testing.assert_array_equal(r["header"][:6], want[0][:6])
    ifg = r["ifg"].cpu().numpy()
    assert rel_err(ifg, want[1]) < 1e-5
    assert phase_rms(ifg, want[1]) < 1e-3
    # amplitude looks and coherence vs the NumPy reference formulas
    box = r["box"]
    a1 = np.sqrt(oc.powlooks(ox.crop(h1, d1, box), rl, cl))
    a2 = np.sqrt(oc.powlooks(ox.crop(h2, d2, box), rl, cl))
    assert rel_err(r["amp1"].cpu().numpy(), a1) < 1e-5
    assert rel_err(r["amp2"].cpu().numpy(), a2) < 1e-5
    _, c = oc.coherence(want[1], a1, a2, seed=0)
    gc = r["coh"].cpu().numpy()
    ok = c <= 1.0 - 1e-5  # pixels whose value is not at the > 1 fill threshold
    assert np.abs(gc[ok] - c[ok]).max() < 1e-4
    assert (gc >= 0).all() and (gc <= 1.0).all()


def test_crossmul_out_float(cuda):
    h1 = formats.make_header(200, 300, 0, 0, 120, 64)
    h2 = formats.make_header(200, 300, 4, 2, 120, 64)
    rng = np.random.default_rng(7)
    d1, d2 = _pair(rng, h1, h2)
    r = interfere.crossmul_pair(h1, torch.from_numpy(d1).to(cuda), h2, torch.from_numpy(d2).to(cuda), 2, 4,
                                out_float=True)
    want = ox.crossmul_pair(h1, d1, h2, d2, 2, 4, out_float=True)
    d = np.angle(np.exp(1j * (r["phase"].cpu().numpy() - want[1])))
    assert np.sqrt(np.mean(d * d)) < 1e-3


def test_crossmul_empty_overlap(cuda):
    h1 = formats.make_header(200, 300, 0, 0, 50, 50)
    h2 = formats.make_header(200, 300, 60, 0, 120, 50)
    z = torch.zeros((50, 50), dtype=torch.complex64, device=cuda)
    z2 = torch.zeros((50, 60), dtype=torch.complex64, device=cuda)
    assert interfere.crossmul_pair(h1, z, h2, z2, 2, 4) is None
    assert ox.crossmul_pair(h1, z.cpu().numpy(), h2, z2.cpu().numpy(), 2, 4) is None


def test_crossmul_union_legacy(cuda):
    h1 = formats.make_header(200, 300, 0, 3, 100, 60)
    h2 = formats.make_header(200, 300, 10, 0, 130, 50)
    rng = np.random.default_rng(9)
    d1, d2 = _pair(rng, h1, h2)
    r = interfere.crossmul_pair(h1, torch.from_numpy(d1).to(cuda), h2, torch.from_numpy(d2).to(cuda), 2, 5,
                                use_union=True, with_coherence=False)
    box = ox.union_box(h1, h2, 2, 5)
    want = ox.crossmul_looks(ox.crop(h1, d1, box), ox.crop(h2, d2, box), 2, 5)
    assert rel_err(r["ifg"].cpu().numpy(), want) < 1e-5


def test_coherence_fill_is_deterministic(cuda):
    """Identical SLCs give coherence ~1; values > 1 are replaced by the seeded fill."""
    h = formats.make_header(64, 64, 0, 0, 64, 32)
    rng = np.random.default_rng(1)
    d = (rng.standard_normal((32, 64)) + 1j * rng.standard_normal((32, 64))).astype(np.complex64)
    t = torch.from_numpy(d).to(cuda)
    a = interfere.crossmul_pair(h, t, h, t, 2, 2, fill_seed=5)["coh"].cpu().numpy()
    b = interfere.crossmul_pair(h, t, h, t, 2, 2, fill_seed=5)["coh"].cpu().numpy()
    np.testing.assert_array_equal(a, b)
    filled = a < 0.999
    if filled.any():
        idx = np.nonzero(filled.ravel())[0]
        np.testing.assert_allclose(a.ravel()[idx], oc.fill_uniform(idx, 5), rtol=0, atol=0)


def test_cc_raster_layout():
    a1 = np.arange(6, dtype=np.float32).reshape(2, 3)
    a2 = np.full((2, 3), 2.0, np.float32)
    c = np.full((2, 3), 0.5, np.float32)
    out = interfere.cc_raster(a1, a2, c)
    np.testing.assert_array_equal(out, oc.cc_rows(a1 * a2, c))
