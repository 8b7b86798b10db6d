"""The amplitude-look, coherence and stitching oracles (oracle/coherence.py,
oracle/stitch.py) against outputs of the reference's own Python
(s1proc/sario.py:397-420, s1proc/coherence.py:14-147,
s1proc/interfere.py:81-180) on seeded inputs (tests/golden/s1proc_pins.npz,
made by tests/golden/make_s1proc_golden.py).  The oracle keeps the
reference's NumPy calls, so the results are identical; the only exception is
the reference's unseeded random fill of coherence values above 1, which the
oracle replaces by a seeded uniform value in [0, 1)."""
import numpy as np

import s1proc_fixture as F
from oracle import coherence as oc
from oracle import stitch as ost


def test_looks_match_reference():
    z = F.load()
    n = 0
    for x, rl, cl, cpx, pw in F.looks_cases(z):
        np.testing.assert_array_equal(oc.cpxlooks(x, rl, cl), cpx)
        np.testing.assert_array_equal(oc.powlooks(x, rl, cl), pw)
        n += 1
    assert n == 5


def test_multilook_matches_reference():
    z = F.load()
    bursts = F.multilook_bursts(z)
    for rl, cl in F.ML_LOOKS:
        np.testing.assert_array_equal(oc.multilook(bursts, rl, cl), z[f"ml_{rl}x{cl}_amp"])


def test_coherence_matches_reference():
    z = F.load()
    ifg, a1, a2, cc, fill = z["coh_ifg"], z["coh_amp1"], z["coh_amp2"], z["coh_cc"], z["coh_fill"]
    prod, c = oc.coherence(ifg, a1, a2, seed=3)
    ncol = ifg.shape[1]
    np.testing.assert_array_equal(prod, cc[:, :ncol])
    assert fill.any() and (~fill).any()
    np.testing.assert_array_equal(c[~fill], cc[:, ncol:][~fill])
    # the fill: a uniform value in [0, 1) on both sides (seeded here, unseeded there)
    for v in (c[fill], cc[:, ncol:][fill]):
        assert (v >= 0).all() and (v < 1).all()
    rows = ~fill.any(1)  # .cc rows without a filled pixel: identical bytes
    np.testing.assert_array_equal(oc.cc_rows(prod, c)[rows], cc[rows])


def test_stitch_matches_reference():
    z = F.load()
    nrow0, ncol0 = (int(v) for v in z["st_shape"])
    frame = ost.stitch(F.stitch_bursts(z), nrow0, ncol0)
    want = z["st_frame"]
    np.testing.assert_array_equal(frame, want)
