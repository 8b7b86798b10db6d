"""Burst stitching on the GPU (libs1b ``s1b_stitch``): the per-burst
interferograms of a frame merged into one raster with the overlap phase
offsets removed, as s1proc/interfere.py:81-180 does on memmaps.

``stitch_bursts`` works on device tensors (e.g. the products of
``BatchedFrameChain``); ``stitch`` mirrors the file-level function: burst
``.int`` files (64-word header + data), subswath from ``iw<k>`` in the path,
the pair of burst ids from the file name words 1+2 and 7+8, the frame written
as a raw raster and the burst files removed, as the reference does.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib, formats


def stitch_bursts(bursts, nrow0, ncol0, out_float=False, return_offsets=False):
    """bursts: [(box (left, top, right, bottom), data [h, w] device tensor
    complex64 (float32 with out_float), subswath 1..3, group int)].
    Returns the frame [nrow0, ncol0] (and the offset applied to each burst)."""
    dtype = torch.float32 if out_float else torch.complex64
    if not bursts:
        raise ValueError("no bursts")
    dev = bursts[0][1].device
    parts, table, off = [], [], 0
    for (l, t, r, b), d, sw, grp in bursts:
        d = d.to(dtype).contiguous()
        if tuple(d.shape) != (b - t, r - l):
            raise ValueError("burst data does not match its box")
        parts.append(d.reshape(-1))
        table.append(_lib.StitchBurst(off, int(l), int(t), int(r), int(b), int(sw), int(grp)))
        off += d.numel()
    data = torch.cat(parts)
    arr = (_lib.StitchBurst * len(table))(*table)
    lib = _lib.load()
    ws_bytes = int(lib.s1b_stitch_workspace_bytes(arr, len(table), 1 if out_float else 0))
    if ws_bytes == 0:
        raise ValueError("bad burst table")
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    frame = torch.empty((nrow0, ncol0), dtype=dtype, device=dev)
    offs = (ctypes.c_double * len(table))() if return_offsets else None
    _lib.check(lib.s1b_stitch(arr, len(table), _lib.dptr(data), 1 if out_float else 0, int(nrow0), int(ncol0),
                              _lib.dptr(frame), offs, _lib.dptr(ws), ws_bytes, _lib.stream_ptr()), "s1b_stitch")
    if return_offsets:
        return frame, list(offs)
    return frame


def _group(path, table):
    w = os.path.basename(path).split("_")
    key = (w[1] + w[2], w[7] + w[8]) if len(w) > 8 else (os.path.basename(path),)
    return table.setdefault(key, len(table))


def stitch(burst_pairs, outfile, out_float=False, remove=True):
    """Frame raster from burst interferogram files (interfere.py:153-180).
    burst_pairs: file names (entries that do not exist are skipped)."""
    dtype = np.float32 if out_float else np.complex64
    bursts, groups = [], {}
    nrow0 = ncol0 = None
    for sw in (1, 2, 3):
        for f in burst_pairs:
            if f"iw{sw}" not in f or not os.path.exists(f):
                continue
            h, d = formats.read_raster(f, dtype=dtype)
            if nrow0 is None:
                nrow0, ncol0 = int(h[0]), int(h[1])
            bursts.append(((int(h[2]), int(h[3]), int(h[4]), int(h[5])), torch.from_numpy(d).cuda(), sw,
                           _group(f, groups)))
    if not bursts:
        return None
    frame = stitch_bursts(bursts, nrow0, ncol0, out_float)
    frame.cpu().numpy().tofile(outfile)
    if remove:
        for f in burst_pairs:
            if os.path.exists(f) and any(f"iw{s}" in f for s in (1, 2, 3)):
                os.remove(f)
    return outfile
