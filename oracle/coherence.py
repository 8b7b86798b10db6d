"""Oracle of the reference amplitude multilook and coherence (NumPy in the reference).

Test infrastructure only (see ``oracle/__init__.py``).

Follows:
  * ``s1proc/sario.py:397-413``   cpxlooks (row sums first, then column sums,
                                  then ``/ collook / rowlook``)
  * ``s1proc/sario.py:416-420``   powlooks
  * ``s1proc/coherence.py:14-55`` multilook (look-aligned grid, first non-zero
                                  burst wins)
  * ``s1proc/coherence.py:109-147`` coherence  ``|ifg| / (amp1+1e-12) / (amp2+1e-12)``
  * ``s1proc/sario.py:387-394``   savec row layout ``[real | imag]``

The reference replaces coherence values > 1 with *unseeded* ``np.random.rand``.
The build replaces them with a deterministic uniform value derived from the
pixel index and a seed (``fill_uniform``); the oracle restates that same
function so both sides agree exactly.
"""
from __future__ import annotations

import numpy as np

MASK64 = (1 << 64) - 1


def cpxlooks(imgbg, rowlook, collook):
    """sario.py:397-413, same NumPy calls (same float32 summation order)."""
    naz, nrg = imgbg.shape
    newnaz = int(np.floor(naz / rowlook))
    newnrg = int(np.floor(nrg / collook))
    imgaz = np.zeros((newnaz, nrg), dtype=imgbg.dtype)
    imgsm = np.zeros((newnaz, newnrg), dtype=imgbg.dtype)
    if rowlook > 1:
        for i in range(newnaz):
            imgaz[i, :] = np.sum(imgbg[i * rowlook:(i + 1) * rowlook, :], axis=0)
    else:
        imgaz = imgbg
    if collook > 1:
        for i in range(newnrg):
            imgsm[:, i] = np.sum(imgaz[:, i * collook:(i + 1) * collook], axis=1)
    else:
        imgsm = imgaz
    return imgsm / collook / rowlook


def powlooks(imgbg, rowlook, collook):
    """sario.py:416-420."""
    if rowlook == 1 and collook == 1:
        return np.abs(imgbg)
    return np.abs(cpxlooks(np.abs(imgbg) ** 2, rowlook, collook))


def amp_looks(header, data, rowlook, collook):
    """The per-burst part of multilook(), coherence.py:31-47.

    Returns (top_sm, bottom_sm, left_sm, right_sm, amp float32)."""
    left, top, right, bottom = int(header[2]), int(header[3]), int(header[4]), int(header[5])
    left_sm = (left + collook - 1) // collook
    top_sm = (top + rowlook - 1) // rowlook
    right_sm = right // collook
    bottom_sm = bottom // rowlook
    row_start = top_sm * rowlook - top
    row_end = bottom_sm * rowlook - top
    col_start = left_sm * collook - left
    col_end = right_sm * collook - left
    amp = np.sqrt(powlooks(data[row_start:row_end, col_start:col_end], rowlook, collook))
    return top_sm, bottom_sm, left_sm, right_sm, amp


def multilook(bursts, rowlook, collook):
    """coherence.py:14-55 on in-memory (header, data) bursts; returns float32 [nrow0/rl, ncol0/cl]."""
    out = None
    for i, (hd, data) in enumerate(bursts):
        t, b, l, r, amp = amp_looks(hd, data, rowlook, collook)
        if out is None:
            out = np.zeros((int(hd[0]) // rowlook, int(hd[1]) // collook), dtype=np.float32)
        if i == 0:
            out[t:b, l:r] = amp
        else:
            old = out[t:b, l:r]
            m = (old == 0) & (amp != 0)
            old[m] = amp[m]
    return out


def splitmix64(x):
    """SplitMix64 finaliser (Steele, Lea, Flood 2014) on Python ints."""
    x = (x + 0x9E3779B97F4A7C15) & MASK64
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
    return z ^ (z >> 31)


def fill_uniform(index, seed):
    """Deterministic stand-in for the reference's ``np.random.rand`` fill:
    ``(splitmix64(seed*2^32 + index) >> 40) * 2^-24`` as float32 in [0, 1)."""
    idx = np.asarray(index, dtype=np.uint64).ravel()
    out = np.empty(idx.shape, dtype=np.float32)
    base = (int(seed) << 32) & MASK64
    for k, v in enumerate(idx.tolist()):
        out[k] = np.float32((splitmix64((base + v) & MASK64) >> 40) * (1.0 / 16777216.0))
    return out


def coherence(ifg, amp1, amp2, seed=0):
    """coherence.py:142-146 on float32 arrays; returns (amp1*amp2, c)."""
    c = np.abs(ifg.astype(np.complex64)) / (amp1.astype(np.float32) + 1e-12) / (amp2.astype(np.float32) + 1e-12)
    c = c.astype(np.float32)
    bad = c > 1
    if bad.any():
        c[bad] = fill_uniform(np.nonzero(bad.ravel())[0], seed)
    return (amp1 * amp2).astype(np.float32), c


def cc_rows(prod, c):
    """savec layout (sario.py:387-394): each row is [prod row | c row], float32."""
    nrow, ncol = c.shape
    out = np.zeros((nrow, 2 * ncol), dtype=np.float32)
    out[:, :ncol] = prod
    out[:, ncol:] = c
    return out

