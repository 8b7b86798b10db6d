"""Oracle of the burst stitching of s1proc/interfere.py:81-180 (stitch_subswath,
stitch) on in-memory burst interferograms.  Test infrastructure only (see
``oracle/__init__.py``).

A burst is (header [nrow0, ncol0, left, top, right, bottom, ...], data,
subswath 1..3, group): ``group`` stands for the reference/secondary burst ids
the reference reads from the file names (interfere.py:92-96); the overlap
phase offset is estimated only when it changes from the previous burst.
"""
from __future__ import annotations

import numpy as np


def _load(h, d, left, top, right, bottom):
    """CroppedImage.load_data: the crop within [left, right) x [top, bottom), zero elsewhere."""
    out = np.zeros((bottom - top, right - left), dtype=d.dtype)
    l0, t0, r0, b0 = (int(v) for v in h[2:6])
    ol, or_ = max(left, l0), min(right, r0)
    ot, ob = max(top, t0), min(bottom, b0)
    if ol < or_ and ot < ob:
        out[ot - top:ob - top, ol - left:or_ - left] = d[ot - t0:ob - t0, ol - l0:or_ - l0]
    return out


def stitch_subswath(bursts, out_float=False):
    """interfere.py:81-150.  bursts: [(header, data, group)] of one subswath.
    Returns (left, top, right, bottom, mosaic, offsets applied per burst)."""
    keys = [int(h[3]) + int(h[5]) for h, _, _ in bursts]
    order = np.argsort(keys, kind="stable")
    bs = [bursts[i] for i in order]
    h0, hl = bs[0][0], bs[-1][0]
    left, top = min(int(h0[2]), int(hl[2])), min(int(h0[3]), int(hl[3]))
    right, bottom = max(int(h0[4]), int(hl[4])), max(int(h0[5]), int(hl[5]))
    mean_phase_diff = 0.0
    prev = None
    offsets = []
    ifg = None
    for i, (h, d, grp) in enumerate(bs):
        if i == 0:
            ifg = _load(h, d, left, top, right, bottom)
            prev = grp
            offsets.append(0.0)
            continue
        bl, bt, br, bb = (int(v) for v in h[2:6])
        old = ifg[bt - top:bb - top, bl - left:br - left]
        new = d.copy()
        if out_float:
            replace = (old == 0) & (new != 0)
        else:
            replace = (old.real == 0) & (new.real != 0)
        overlap = None
        if grp != prev:
            overlap = (old != 0) & (new != 0) if out_float else (old.real != 0) & (new != 0)
        prev = grp
        if overlap is not None and np.any(overlap):
            if out_float:
                pd = np.exp(1j * (-old[overlap] + new[overlap]))
            else:
                pd = np.conj(old[overlap]) * new[overlap]
            mean_phase_diff = np.angle(np.mean(pd))
            pd = pd * np.exp(-1j * mean_phase_diff)
            mean_phase_diff += np.median(np.angle(pd))
        if mean_phase_diff != 0:
            if out_float:
                new = new - mean_phase_diff
                new[new > np.pi] -= 2 * np.pi
                new[new < -np.pi] += 2 * np.pi
            else:
                new = new * np.exp(-1j * mean_phase_diff)
        old[replace] = new[replace]
        offsets.append(float(mean_phase_diff))
    return left, top, right, bottom, ifg, offsets


def stitch(bursts, nrow0, ncol0, out_float=False):
    """interfere.py:153-180: subswaths 1..3 stitched, then written into the
    frame in that order where the subswath mosaic is non-zero.
    bursts: [(header, data, subswath, group)]."""
    frame = np.zeros((nrow0, ncol0), dtype=np.float32 if out_float else np.complex64)
    for sw in (1, 2, 3):
        bs = [(h, d, g) for h, d, s, g in bursts if s == sw]
        if not bs:
            continue
        left, top, right, bottom, m, _ = stitch_subswath(bs, out_float)
        old = frame[top:bottom, left:right]
        rep = (m != 0) if out_float else (m.real != 0)
        old[rep] = m[rep]
    return frame
