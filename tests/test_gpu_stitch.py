"""Burst stitching (s1b_stitch) against the oracle restatement of
s1proc/interfere.py:81-180 (oracle/stitch.py): per-burst phase offsets
(mean + median over the overlap), the frame raster, complex and phase
modes, offsets carried over bursts without an overlap."""
import numpy as np
import pytest
import torch

from helpers import phase_rms
from oracle import stitch as ost
from sentinel_gpu_processor_b200 import formats
from sentinel_gpu_processor_b200.stitch import stitch, stitch_bursts

pytestmark = pytest.mark.gpu


def _frame_bursts(seed, nrow0=220, ncol0=300, out_float=False):
    """2 subswaths x 4 bursts with 12-row overlaps, random phase offsets per
    burst, speckle-like amplitudes and a little phase noise; the last burst
    of subswath 2 repeats the previous group (no offset estimate)."""
    rng = np.random.default_rng(seed)
    truth = np.exp(1j * rng.uniform(-np.pi, np.pi, (nrow0, ncol0)))
    out = []
    for sw, (l0, r0) in ((1, (5, 160)), (2, (140, 295))):
        top = 3 + sw
        for k in range(4):
            h = 55 + 3 * k
            l, r = l0 + k % 2, r0 - (k % 3)
            t, b = top, min(top + h, nrow0)
            off = rng.uniform(-np.pi, np.pi)
            amp = rng.rayleigh(1.0, (b - t, r - l))
            noise = np.exp(1j * rng.normal(0, 0.2, (b - t, r - l)))
            d = (amp * truth[t:b, l:r] * noise * np.exp(1j * off)).astype(np.complex64)
            d[:, :3] = 0  # ragged edges
            d[rng.random(d.shape) < 0.02] = 0
            grp = sw * 10 + (k if not (sw == 2 and k == 3) else 2)
            if out_float:
                d = np.where(d != 0, np.angle(d), 0).astype(np.float32)
            out.append((formats.make_header(nrow0, ncol0, l, t, r, b), d, sw, grp))
            top = b - 12
    return out, nrow0, ncol0


@pytest.mark.parametrize("out_float", [False, True])
def test_stitch_matches_oracle(cuda, out_float):
    bursts, nrow0, ncol0 = _frame_bursts(3, out_float=out_float)
    want = ost.stitch(bursts, nrow0, ncol0, out_float)
    dev = [((int(h[2]), int(h[3]), int(h[4]), int(h[5])), torch.from_numpy(d).to(cuda), sw, g)
           for h, d, sw, g in bursts]
    got, offs = stitch_bursts(dev, nrow0, ncol0, out_float, return_offsets=True)
    got = got.cpu().numpy()
    # offsets per burst: the oracle's, in each subswath's sorted order
    for sw in (1, 2):
        bs = [(h, d, g) for h, d, s, g in bursts if s == sw]
        _, _, _, _, _, want_off = ost.stitch_subswath(bs, out_float)
        got_sw = [o for (h, d, s, g), o in zip(bursts, offs) if s == sw]
        keys = [int(h[3]) + int(h[5]) for h, d, g in bs]
        got_sorted = [got_sw[i] for i in np.argsort(keys, kind="stable")]
        d = np.angle(np.exp(1j * (np.array(got_sorted) - np.array(want_off))))
        assert np.abs(d).max() < 1e-4
    assert np.array_equal(got != 0, want != 0)
    if out_float:
        d = np.angle(np.exp(1j * (got.astype(np.float64) - want)))
        assert np.abs(d).max() < 1e-3
    else:
        assert phase_rms(got, want) < 1e-4
        assert np.abs(np.abs(got) - np.abs(want)).max() < 1e-4 * np.abs(want).max()


def test_stitch_files_mirror(cuda, tmp_path):
    bursts, nrow0, ncol0 = _frame_bursts(8)
    files = []
    for i, (h, d, sw, g) in enumerate(bursts):
        # s1proc names: words 1+2 and 7+8 identify the reference / secondary bursts
        f = str(tmp_path / f"S1_r{g}_x_iw{sw}_a_b_c_s{g}_y_iw{sw}.int")
        if f in files:
            f = f.replace(".int", f"_{i}.int")
        formats.write_raster(f, h, d)
        files.append(f)
    out = str(tmp_path / "frame.int")
    assert stitch(files, out) == out
    got = np.fromfile(out, dtype=np.complex64).reshape(nrow0, ncol0)
    want = ost.stitch(bursts, nrow0, ncol0)
    assert np.array_equal(got != 0, want != 0)
    assert phase_rms(got, want) < 1e-4
    assert not any(__import__("os").path.exists(f) for f in files)  # burst files removed, as the reference does
