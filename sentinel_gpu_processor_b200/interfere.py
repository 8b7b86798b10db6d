"""Interferogram formation: the in-process equivalent of one
``crossmul_daemon`` task (csrc/src/crossmul_daemon.cu:566-975) plus the
amplitude multilook and coherence of s1proc/coherence.py, fused.
"""
from __future__ import annotations

import os

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


# ----------------------------------------------------------------------------
# s1proc's interfere() call surface (s1proc/interfere.py:536-704)
# ----------------------------------------------------------------------------

def _subswaths(burst_files):
    """Burst files of one date grouped by subswath (``iw1``..``iw3`` in the
    name) and sorted by top + bottom of their crop, as sario.BurstGroup /
    Subswath do (s1proc/sario.py:218-266).  Returns [[(path, header)], x3]."""
    out = []
    for sw in range(1, 4):
        bs = []
        for f in burst_files:
            if f"iw{sw}" in f:
                bs.append((f, formats.read_header(f)))
        bs.sort(key=lambda b: int(b[1][3]) + int(b[1][5]))
        out.append(bs)
    return out


def match_bursts(ref_bursts, sec_bursts):
    """For every reference burst the secondary burst of the nearest crop
    rows (|top difference| + |bottom difference|, first minimum), as
    s1proc/interfere.py:17-45.  Bursts: [(path, header)]."""
    if not ref_bursts or not sec_bursts:
        return []
    tops = np.array([int(h[3]) for _, h in sec_bursts])
    bottoms = np.array([int(h[5]) for _, h in sec_bursts])
    pairs = []
    for f, h in ref_bursts:
        k = int(np.argmin(np.abs(tops - int(h[3])) + np.abs(bottoms - int(h[5]))))
        pairs.append((f, sec_bursts[k][0]))
    return pairs


def burst_pair_tasks(ref_files, sec_files, ifg_path):
    """(ref, sec, out) burst-pair tasks of one date pair, subswath by
    subswath, the output named <ref burst>_<sec burst>.int in ``ifg_path``
    (s1proc/interfere.py:48-78, 183-210)."""
    tasks = []
    for rb, sb in zip(_subswaths(ref_files), _subswaths(sec_files)):
        for f1, f2 in match_bursts(rb, sb):
            n1 = os.path.splitext(os.path.basename(f1))[0]
            n2 = os.path.splitext(os.path.basename(f2))[0]
            tasks.append((f1, f2, os.path.join(ifg_path, n1 + "_" + n2 + ".int")))
    return tasks


def check_tuning(io_workers=-1, cpu_workers=-1, gpu_workers=-1, streams_per_gpu=-1, max_slots=-1):
    """The daemon's all-or-nothing tuning contract (s1proc/interfere.py:642-663):
    every value -1 (automatic) or every value a positive int; anything else
    prints the reference's fatal message and exits with status 1."""
    vals = (io_workers, cpu_workers, gpu_workers, streams_per_gpu, max_slots)
    if all(v == -1 for v in vals) or all(isinstance(v, int) and v > 0 for v in vals):
        return
    import sys
    print("[FATAL] Invalid parameter configuration. Please either omit all tuning arguments for hardware-managed "
          "auto-tuning, or provide the complete set of parameters (--io-workers, --cpu-workers, --streams-per-gpu, "
          "--gpu-workers, --max-slots). Partial overrides are not allowed.", file=sys.stderr)
    raise SystemExit(1)


def interfere(img_pair_file: str, slc_path: str, rscfile: str, small_rsc_file: str, ifg_path: str = "igrams",
              rowlook: int = 1, collook: int = 1, out_float: bool = False, io_workers: int = -1,
              cpu_workers: int = -1, gpu_workers: int = -1, streams_per_gpu: int = -1, max_slots: int = -1,
              verbose: bool = False):
    """Interferograms of the date pairs listed in ``ifg_path/img_pair_file``
    (lines ``<ref date> <sec date>``) from the geocoded bursts
    ``slc_path/<date>*.gslc``: the multilooked RSC written to
    ``small_rsc_file``, burst pairs matched per subswath, crossmul + looks on
    the GPU for every burst pair whose output is missing, then the burst
    interferograms stitched into ``ifg_path/<ref>_<sec>.int`` (raw, frame
    grid) with the burst files removed.  Same arguments, files and
    behaviour as s1proc/interfere.py:536-704; the daemon's host-pipeline
    tuning arguments are checked the same way and otherwise unused (the
    burst pairs run in-process on the GPU).  Returns (ok, failed)."""
    import glob

    from . import stitch as _stitch
    os.makedirs(ifg_path, exist_ok=True)
    rsc = formats.read_rsc(rscfile)
    if os.path.dirname(small_rsc_file):
        os.makedirs(os.path.dirname(small_rsc_file), exist_ok=True)
    formats.write_rsc(small_rsc_file, rsc.take_look(rowlook, collook))
    pairs, groups = [], {}
    with open(os.path.join(ifg_path, img_pair_file)) as f:
        for line in f:
            w = line.split()
            if len(w) < 2:
                continue
            pairs.append((w[0], w[1]))
            for d in w[:2]:
                if d not in groups:
                    groups[d] = glob.glob(os.path.join(slc_path, f"{d}*.gslc"))
    tasks, frame_map = [], {}
    for ref, sec in pairs:
        outfile = os.path.join(ifg_path, f"{ref}_{sec}.int")
        if os.path.exists(outfile):
            continue
        t = burst_pair_tasks(groups[ref], groups[sec], ifg_path)
        frame_map[outfile] = [x[2] for x in t]
        if not all(os.path.exists(x[2]) for x in t):
            tasks.extend(t)
    if not tasks:
        for outfile, parts in frame_map.items():
            _stitch.stitch(parts, outfile, out_float)
        return 0, 0
    check_tuning(io_workers, cpu_workers, gpu_workers, streams_per_gpu, max_slots)
    todo = [t for t in tasks if not os.path.exists(t[2])]
    emit = print if verbose else (lambda *a, **k: None)
    ok, failed = crossmul_files(todo, rowlook, collook, out_float=out_float, emit=emit)
    for outfile, parts in frame_map.items():
        _stitch.stitch(parts, outfile, out_float)
    return ok, failed
