"""s1proc's coherence call surface on the GPU (s1proc/coherence.py:14-147):
``multilook`` (amplitude mosaic of one date's geocoded bursts, ``.amp``),
``multilook_amp`` (every date of a directory) and ``coherence`` (``.cc``
rasters of stitched interferograms), with the same names, arguments and
files.  Amplitude looks and coherence run in libs1b kernels
(``s1b_amp_looks``, ``s1b_coherence_cc``).

Coherence values above 1 are replaced by a uniform [0, 1) value of (seed,
pixel index) where s1proc draws unseeded ``np.random.rand``: the same
distribution, reproducible.
"""
from __future__ import annotations

import glob
import os
from typing import Sequence

import numpy as np
import torch

from . import formats, kernels


def multilook(slc_list: Sequence[str], outfile: str, rowlook: int, collook: int):
    """Amplitude mosaic of geocoded SLCs (``.gslc``) on the frame grid of the
    first one: sqrt of the rl x cl mean power, the first image written whole,
    later ones only where the mosaic is still 0 (s1proc/coherence.py:14-55)."""
    amp = None
    for i, path in enumerate(slc_list):
        h, d = formats.read_raster(path)
        nrow0, ncol0, left, top = (int(v) for v in h[:4])
        if amp is None:
            amp = torch.zeros((nrow0 // rowlook, ncol0 // collook), dtype=torch.float32, device="cuda")
        kernels.amp_looks(torch.from_numpy(np.ascontiguousarray(d)).cuda(), left, top, nrow0, ncol0, rowlook, collook,
                          first=(i == 0), amp=amp)
    if amp is not None:
        amp.cpu().numpy().tofile(outfile)


def multilook_amp(slc_dir: str, amp_dir: str = "amp", rowlook: int = 1, collook: int = 1):
    """``<date>.amp`` for every date of ``slc_dir``'s ``*.gslc`` (date = the
    first 8 characters of the file name); existing outputs are kept
    (s1proc/coherence.py:58-83)."""
    os.makedirs(amp_dir, exist_ok=True)
    slc_list = glob.glob(os.path.join(slc_dir, "*.gslc"))
    for date in sorted({os.path.basename(s)[0:8] for s in slc_list}):
        outfile = os.path.join(amp_dir, f"{date}.amp")
        if os.path.exists(outfile):
            continue
        multilook(glob.glob(os.path.join(slc_dir, f"{date}*.gslc")), outfile, rowlook, collook)


def coherence(ifg_dir: str, amp_dir: str, nrow: int, ncol: int, rowlook: int, collook: int, fill_seed: int = 0):
    """``.cc`` beside every ``*.int`` of ``ifg_dir`` (raw complex64 nrow x ncol,
    named ``<date1>_<date2>...``): rows [amp1*amp2 | coherence] with the
    dates' ``.amp`` (s1proc/coherence.py:109-147)."""
    os.makedirs(amp_dir, exist_ok=True)
    cache = {}

    def amp(date):
        if date not in cache:
            a = np.fromfile(os.path.join(amp_dir, f"{date}.amp"), dtype=np.float32).reshape(nrow, ncol)
            if len(cache) > 8:
                cache.clear()
            cache[date] = torch.from_numpy(a).cuda()
        return cache[date]

    for ifg_file in sorted(glob.glob(os.path.join(ifg_dir, "*.int"))):
        base = os.path.basename(ifg_file)
        ifg = np.fromfile(ifg_file, dtype=np.complex64).reshape(nrow, ncol)
        cc = kernels.coherence_cc(torch.from_numpy(ifg).cuda(), amp(base[0:8]), amp(base[9:17]), fill_seed)
        cc.cpu().numpy().tofile(ifg_file.replace(".int", ".cc"))
