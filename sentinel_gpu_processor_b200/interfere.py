"""Interferogram formation: the in-process equivalent of one
``crossmul_daemon`` task (csrc/src/crossmul_daemon.cu:566-975) plus the
amplitude multilook and coherence of s1proc/coherence.py, fused.
"""
from __future__ import annotations

import numpy as np
import torch

from . import formats, kernels, plan as _plan


def crossmul_pair(h1, d1: torch.Tensor, h2, d2: torch.Tensor, rowlook: int, collook: int,
                  out_float: bool = False, with_coherence: bool = True, fill_seed: int = 0,
                  use_union: bool = False):
    """One burst pair.

    h1/h2: ``.gslc`` headers (>= 6 int32), d1/d2: complex64 CUDA tensors of
    the cropped rasters.  Returns None for an empty overlap (the daemon's
    FAIL ``empty overlap region``), else a dict with ``header`` (int32[64]),
    ``ifg`` (complex64) or ``phase`` (float32, when ``out_float``), and
    ``amp1``, ``amp2``, ``coh`` when ``with_coherence``.
    """
    box, hdr6 = _plan.crossmul_box(h1, h2, rowlook, collook, use_union)
    if box is None:
        return None
    hdr = formats.make_header(*hdr6)
    if use_union:
        # legacy crossmul: zero-filled union grid (read_and_resample, sario.hpp:141-225)
        d1 = _pad_to(h1, d1, box)
        d2 = _pad_to(h2, d2, box)
        b1 = b2 = (box[0], box[1])
    else:
        b1 = (int(h1[2]), int(h1[3]))
        b2 = (int(h2[2]), int(h2[3]))
    want = ["phase"] if out_float else ["ifg"]
    if with_coherence:
        want += ["amp1", "amp2", "coh"]
    outs = kernels.crossmul_looks(d1, b1, d2, b2, box, rowlook, collook, want=tuple(want), fill_seed=fill_seed)
    outs["header"] = hdr
    outs["box"] = box
    return outs


def _pad_to(h, d, box):
    left, top, right, bottom = box
    out = torch.zeros((bottom - top, right - left), dtype=d.dtype, device=d.device)
    l0, t0, r0, b0 = int(h[2]), int(h[3]), int(h[4]), int(h[5])
    ol, or_ = max(left, l0), min(right, r0)
    ot, ob = max(top, t0), min(bottom, b0)
    if ol < or_ and ot < ob:
        out[ot - top:ob - top, ol - left:or_ - left] = d[ot - t0:ob - t0, ol - l0:or_ - l0]
    return out


def crossmul_files(tasks, rowlook, collook, out_float=False, emit=print):
    """File-level drop-in for the daemon: ``tasks`` = [(ref, sec, out)] paths.

    Writes each output raster, emits ``OK <out>`` per success and a final
    ``SUMMARY ok failed total seconds`` line (crossmul_daemon.cu:1171,
    1897-1899); failures are reported as ``FAIL <out> - reason`` and do not
    stop the run.  Returns (ok, failed).
    """
    import sys
    import time
    t0 = time.time()
    ok = failed = 0
    for ref, sec, out in tasks:
        try:
            h1, d1 = formats.read_raster(ref)
            h2, d2 = formats.read_raster(sec)
            r = crossmul_pair(h1, torch.from_numpy(d1).cuda(), h2, torch.from_numpy(d2).cuda(), rowlook, collook,
                              out_float=out_float, with_coherence=False)
            if r is None:
                print(f"[crossmul_daemon] FAIL {out} - empty overlap region", file=sys.stderr)
                failed += 1
                continue
            data = r["phase"] if out_float else r["ifg"]
            formats.write_raster(out, r["header"], data.cpu().numpy())
            emit(f"OK {out}")
            ok += 1
        except (OSError, IOError, ValueError) as e:
            print(f"[crossmul_daemon] FAIL {out} - I/O error: {e}", file=sys.stderr)
            failed += 1
    emit(f"SUMMARY {ok} {failed} {len(tasks)} {int(time.time() - t0)}")
    return ok, failed


def cc_raster(amp1: np.ndarray, amp2: np.ndarray, coh: np.ndarray) -> np.ndarray:
    """``.cc`` rows ``[amp1*amp2 | coherence]`` (s1proc/coherence.py:145-147, sario.py:387-394)."""
    nrow, ncol = coh.shape
    out = np.empty((nrow, 2 * ncol), dtype=np.float32)
    out[:, :ncol] = amp1.astype(np.float32) * amp2.astype(np.float32)
    out[:, ncol:] = coh
    return out
