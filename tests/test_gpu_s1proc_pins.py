"""The GPU amplitude looks, coherence and stitching (s1proc's call surface in
coherence.py and stitch.py, libs1b kernels underneath) against outputs of
the reference's own Python (tests/golden/s1proc_pins.npz, made by
tests/golden/make_s1proc_golden.py from s1proc/coherence.py:14-147,
s1proc/sario.py:397-420 and s1proc/interfere.py:81-180).  The files are
written and read in the reference's formats.

Tolerances: amplitudes and coherence within 2e-6 relative (float32 sums in
another order), the coherence fill (values above 1) in [0, 1) on both sides;
stitched frame: identical zero pattern, values within 1e-5 (the overlap
phase offset is estimated in float64 here, in complex64 NumPy there).
"""
import os

import numpy as np
import pytest
import torch

import s1proc_fixture as F
from helpers import phase_rms
from sentinel_gpu_processor_b200 import coherence as C
from sentinel_gpu_processor_b200 import kernels, stitch as ST

pytestmark = pytest.mark.gpu


def _write(path, h, d):
    with open(path, "wb") as f:
        np.asarray(h, dtype=np.int32).tofile(f)
        np.ascontiguousarray(d).tofile(f)


def test_multilook_files_match_reference(cuda, tmp_path):
    z = F.load()
    files = []
    for i, (h, d) in enumerate(F.multilook_bursts(z)):
        hd = np.zeros(64, dtype=np.int32)
        hd[:6] = h[:6]
        f = str(tmp_path / f"20200101_S1A_AAAA_iw1_burst_{i}.gslc")
        _write(f, hd, d)
        files.append(f)
    for rl, cl in F.ML_LOOKS:
        out = str(tmp_path / f"m{rl}x{cl}.amp")
        C.multilook(files, out, rl, cl)
        want = z[f"ml_{rl}x{cl}_amp"]
        got = np.fromfile(out, dtype=np.float32).reshape(want.shape)
        np.testing.assert_array_equal(got > 0, want > 0)
        assert np.abs(got - want).max() <= 2e-6 * want.max()


def test_coherence_files_match_reference(cuda, tmp_path):
    z = F.load()
    ifg, a1, a2, cc, fill = z["coh_ifg"], z["coh_amp1"], z["coh_amp2"], z["coh_cc"], z["coh_fill"]
    nrow, ncol = ifg.shape
    (tmp_path / "ifg").mkdir()
    (tmp_path / "amp").mkdir()
    ifg.tofile(str(tmp_path / "ifg" / "20200101_20200113.int"))
    a1.tofile(str(tmp_path / "amp" / "20200101.amp"))
    a2.tofile(str(tmp_path / "amp" / "20200113.amp"))
    C.coherence(str(tmp_path / "ifg"), str(tmp_path / "amp"), nrow, ncol, 2, 4)
    got = np.fromfile(str(tmp_path / "ifg" / "20200101_20200113.cc"), dtype=np.float32).reshape(nrow, 2 * ncol)
    assert np.abs(got[:, :ncol] - cc[:, :ncol]).max() <= 2e-6 * cc[:, :ncol].max()
    gc, wc = got[:, ncol:], cc[:, ncol:]
    assert np.abs(gc[~fill] - wc[~fill]).max() <= 2e-6
    assert (gc[fill] >= 0).all() and (gc[fill] < 1).all()
    # the same through the kernel entry point
    k = kernels.coherence_cc(torch.from_numpy(ifg).to(cuda), torch.from_numpy(a1).to(cuda),
                             torch.from_numpy(a2).to(cuda)).cpu().numpy()
    np.testing.assert_array_equal(k, got)


def test_stitch_files_match_reference(cuda, tmp_path):
    z = F.load()
    names = [str(n) for n in z["st_names"]]
    paths = []
    for k, name in enumerate(names):
        hd = np.zeros(64, dtype=np.int32)
        hd[:6] = z[f"st_burst{k}_hdr"][:6]
        p = str(tmp_path / name)
        _write(p, hd, z[f"st_burst{k}_data"])
        paths.append(p)
    out = str(tmp_path / "frame.int")
    ST.stitch(paths, out, False)
    want = z["st_frame"]
    got = np.fromfile(out, dtype=np.complex64).reshape(want.shape)
    np.testing.assert_array_equal(np.abs(got) > 0, np.abs(want) > 0)
    assert np.abs(got - want).max() < 1e-5
    assert phase_rms(got, want) < 1e-5
    assert not any(os.path.exists(p) for p in paths)  # burst files removed, as the reference does
