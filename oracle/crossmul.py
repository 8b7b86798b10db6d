"""Oracle of the reference crossmul + multilook (``crossmul_daemon`` / ``crossmul``).

Test infrastructure only (see ``oracle/__init__.py``).

Follows:
  * ``csrc/src/crossmul_daemon.cu:612-666``  intersection box aligned to looks,
    output header ``[nrow0/rl, ncol0/cl, left/cl, top/rl, right/cl, bottom/rl]``
  * ``csrc/src/crossmul.cu:191-213``         legacy union box
  * ``csrc/src/crossmul_daemon.cu:520-528``  crop of each SLC to the box
  * ``csrc/src/sario.cu:199-211``            conj_mul  c = conj(a) * b
  * ``csrc/src/sario.cu:241-262``            cpx_col_look (sequential sum / collook)
  * ``csrc/src/sario.cu:264-286``            cpx_row_look (sequential sum / rowlook)
  * ``csrc/src/sario.cu:231-239``            point_angle (atan2f)
All arithmetic is float32 in the reference's summation order.
"""
from __future__ import annotations

import numpy as np


def intersection_box(h1, h2, rowlook, collook):
    """crossmul_daemon.cu:612-620 -> (left, top, right, bottom) or None if empty."""
    left = max(int(h1[2]), int(h2[2]))
    left = (left + collook - 1) // collook * collook
    right = min(int(h1[4]), int(h2[4]))
    right = right // collook * collook
    top = max(int(h1[3]), int(h2[3]))
    top = (top + rowlook - 1) // rowlook * rowlook
    bottom = min(int(h1[5]), int(h2[5]))
    bottom = bottom // rowlook * rowlook
    if bottom - top <= 0 or right - left <= 0:
        return None
    return left, top, right, bottom


def union_box(h1, h2, rowlook, collook):
    """crossmul.cu:191-206 (legacy executable) -> box or None if empty."""
    left = min(int(h1[2]), int(h2[2]))
    left = (left + collook - 1) // collook * collook
    right = max(int(h1[4]), int(h2[4]))
    right = right // collook * collook
    top = min(int(h1[3]), int(h2[3]))
    top = (top + rowlook - 1) // rowlook * rowlook
    bottom = max(int(h1[5]), int(h2[5]))
    bottom = bottom // rowlook * rowlook
    if (bottom - top) // rowlook == 0 or (right - left) // collook == 0:
        return None
    return left, top, right, bottom


def ifg_header(h1, box, rowlook, collook):
    """crossmul_daemon.cu:660-666."""
    left, top, right, bottom = box
    hd = np.zeros(64, dtype=np.int32)
    hd[0] = int(h1[0]) // rowlook
    hd[1] = int(h1[1]) // collook
    hd[2] = left // collook
    hd[3] = top // rowlook
    hd[4] = right // collook
    hd[5] = bottom // rowlook
    return hd


def crop(header, data, box):
    """Cut ``box`` out of a cropped image; pixels outside the image are zero
    (the daemon reads only the intersection; ``read_and_resample`` zero-fills)."""
    left, top, right, bottom = box
    out = np.zeros((bottom - top, right - left), dtype=data.dtype)
    l0, t0, r0, b0 = int(header[2]), int(header[3]), int(header[4]), int(header[5])
    ol, or_ = max(left, l0), min(right, r0)
    ot, ob = max(top, t0), min(bottom, b0)
    if ol < or_ and ot < ob:
        out[ot - top:ob - top, ol - left:or_ - left] = data[ot - t0:ob - t0, ol - l0:or_ - l0]
    return out


def conj_mul(a, b):
    """sario.cu:199-211 in float32."""
    ax, ay = a.real.astype(np.float32), a.imag.astype(np.float32)
    bx, by = b.real.astype(np.float32), b.imag.astype(np.float32)
    out = np.empty(a.shape, dtype=np.complex64)
    out.real = ax * bx + ay * by
    out.imag = -ay * bx + ax * by
    return out


def col_look(a, collook):
    """cpx_col_look, sario.cu:241-262: sequential float32 sum over collook, / collook."""
    nrow, ncol = a.shape
    ncs = ncol // collook
    v = a[:, :ncs * collook].reshape(nrow, ncs, collook)
    sr = np.zeros((nrow, ncs), dtype=np.float32)
    si = np.zeros((nrow, ncs), dtype=np.float32)
    for j in range(collook):
        sr = sr + v[:, :, j].real
        si = si + v[:, :, j].imag
    out = np.empty((nrow, ncs), dtype=np.complex64)
    out.real = sr / np.float32(collook)
    out.imag = si / np.float32(collook)
    return out


def row_look(a, rowlook):
    """cpx_row_look, sario.cu:264-286: sequential float32 sum over rowlook, / rowlook."""
    nrow, ncol = a.shape
    nrs = nrow // rowlook
    v = a[:nrs * rowlook].reshape(nrs, rowlook, ncol)
    sr = np.zeros((nrs, ncol), dtype=np.float32)
    si = np.zeros((nrs, ncol), dtype=np.float32)
    for j in range(rowlook):
        sr = sr + v[:, j].real
        si = si + v[:, j].imag
    out = np.empty((nrs, ncol), dtype=np.complex64)
    out.real = sr / np.float32(rowlook)
    out.imag = si / np.float32(rowlook)
    return out


def crossmul_looks(ref, sec, rowlook, collook):
    """conj_mul -> col look (if >1) -> row look (if >1).  crossmul_daemon.cu:921-956."""
    ifg = conj_mul(ref, sec)
    if collook > 1:
        ifg = col_look(ifg, collook)
    if rowlook > 1:
        ifg = row_look(ifg, rowlook)
    return ifg


def point_angle(z):
    """sario.cu:231-239."""
    return np.arctan2(z.imag.astype(np.float32), z.real.astype(np.float32)).astype(np.float32)


def crossmul_pair(h1, d1, h2, d2, rowlook, collook, out_float=False):
    """One daemon task (crossmul_daemon.cu:566-975): returns (header, data) or None."""
    box = intersection_box(h1, h2, rowlook, collook)
    if box is None:
        return None
    ref = crop(h1, d1, box)
    sec = crop(h2, d2, box)
    ifg = crossmul_looks(ref, sec, rowlook, collook)
    hd = ifg_header(h1, box, rowlook, collook)
    return hd, (point_angle(ifg) if out_float else ifg)
