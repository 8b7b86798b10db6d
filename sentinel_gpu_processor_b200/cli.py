"""Command-line drop-ins for the reference executables, with their names,
arguments, stdout lines, exit codes and files, so that s1proc finds them
through ``get_bin_path`` unchanged (the stubs in ``bin/``):

    geo2rdr dbname slcoutfile [slcinfile] [--stdin] [--gpu N]          geo2rdr.cu:704-734
            [--tiff FILE[::MEMBER]]  (extension: bursts straight from the
            measurement TIFF, or a member of the SAFE zip, instead of the
            pipe s1proc/sentinel_scene.py:164-207, 419-437 feeds)
    crossmul_daemon --rowlook R --collook C [--out-float] [--verbose]
                    --tasks-file F [--io-workers .. --max-slots]       crossmul_daemon.cu:1744-1911
    crossmul input_file rowlook collook out_float [--gpu N]            crossmul.cu:285-298
    goldstein in_str nrow ncol n_win alpha [out_str] [--gpu N]         goldstein.cu:504-524

The work is done by the s1b library on one GPU.  The daemon's host pipeline
tuning arguments are accepted and validated (all or none, as the reference
demands) but have no effect: tasks run one after the other on the device.
"""
from __future__ import annotations

import os
import sys
import time

import numpy as np

USAGE_GEO2RDR = ("Usage: geo2rdr dbname slcoutfile [slcinfile] [--stdin] [--gpu DEVICE_ID]\n"
                 "  --stdin  Read original SLC burst data from stdin")
# Extension of this build (not printed, so the usage text stays the reference's):
#   --tiff FILE[::MEMBER]  read the bursts from a measurement TIFF (or a member of a zip)
USAGE_CROSSMUL = "Usage: crossmul input_file rowlook collook out_float [--gpu DEVICE_ID]"
USAGE_GOLDSTEIN = "Usage: goldstein in_str nrow ncol n_win alpha [out_str] [--gpu DEVICE_ID]"
TUNING = ("--io-workers", "--cpu-workers", "--streams-per-gpu", "--gpu-workers", "--max-slots")


def _gpu_arg(argv):
    """``--gpu N`` / ``-g N`` anywhere after the program name (gpu_device.hpp:71-79); -1 if absent."""
    for i in range(1, len(argv) - 1):
        if argv[i] in ("--gpu", "-g"):
            return int(argv[i + 1])
    return -1


def _set_gpu(argv):
    dev = _gpu_arg(argv)
    if dev >= 0:
        import torch
        torch.cuda.set_device(dev)


def _get_arg(argv, name, default):
    for i in range(1, len(argv) - 1):
        if argv[i] == name:
            return argv[i + 1]
    return default


def geo2rdr_main(argv=None, stdin=None):
    argv = list(sys.argv if argv is None else argv)
    use_stdin = "--stdin" in argv[1:]
    if len(argv) < 3:
        print(USAGE_GEO2RDR)
        return 0
    _set_gpu(argv)
    db, out = argv[1], argv[2]
    slcin = None
    if len(argv) > 3 and argv[3] not in ("--stdin", "--gpu", "-g", "--tiff"):
        slcin = argv[3]
    tiff_arg = _get_arg(argv, "--tiff", None)
    from .geo2rdr import geo2rdr_files
    try:
        if tiff_arg is not None:
            from .ingest import MeasurementTiff
            path, _, member = tiff_arg.partition("::")
            with MeasurementTiff(path, member or None) as tif:
                geo2rdr_files(db, out, tiff=tif)
        else:
            geo2rdr_files(db, out, slcin, stream=(stdin or sys.stdin.buffer) if use_stdin else None)
    except (EOFError, ValueError, OSError, KeyError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    return 0


def read_tasks(path):
    """``ref sec out`` per line; blank lines skipped, malformed ones warned
    about (crossmul_daemon.cu:1499-1525)."""
    tasks = []
    with open(path) as f:
        for line in f:
            if not line.strip():
                continue
            parts = line.split()
            if len(parts) >= 3:
                tasks.append(tuple(parts[:3]))
            else:
                print(f"[crossmul_daemon] WARNING: skipping malformed task line: {line.rstrip()}", file=sys.stderr)
    return tasks


def crossmul_daemon_main(argv=None, emit=print):
    argv = list(sys.argv if argv is None else argv)
    rowlook = int(_get_arg(argv, "--rowlook", "1"))
    collook = int(_get_arg(argv, "--collook", "1"))
    out_float = "--out-float" in argv[1:]
    tuning = [int(_get_arg(argv, k, "-1")) for k in TUNING]
    all_auto = all(v == -1 for v in tuning)
    all_manual = all(v > 0 for v in tuning)
    if not all_auto and not all_manual:
        print("[FATAL] Invalid parameter configuration. Please either omit all tuning arguments for "
              "hardware-managed auto-tuning, or provide the complete set of parameters (--io-workers, "
              "--cpu-workers, --streams-per-gpu, --gpu-workers, --max-slots). Partial overrides are not allowed.",
              file=sys.stderr)
        return 1
    tasks_file = _get_arg(argv, "--tasks-file", "")
    if not tasks_file:
        print("[crossmul_daemon] ERROR: --tasks-file <path> is required.", file=sys.stderr)
        return 1
    if not os.path.isfile(tasks_file):
        print(f"[crossmul_daemon] ERROR: cannot open tasks file: {tasks_file}", file=sys.stderr)
        tasks = []
    else:
        tasks = read_tasks(tasks_file)
    if not tasks:
        print("[crossmul_daemon] No tasks found in file.  Exiting.", file=sys.stderr)
        return 0
    print(f"[crossmul_daemon] Loaded {len(tasks)} tasks.", file=sys.stderr)
    from .interfere import crossmul_files
    t0 = time.time()
    ok, failed = crossmul_files(tasks, rowlook, collook, out_float=out_float,
                                emit=lambda s: emit(s) if not s.startswith("SUMMARY") else None)
    emit(f"PROGRESS {ok} {failed} {len(tasks)} {int(time.time() - t0)}")
    emit(f"SUMMARY {ok} {failed} {len(tasks)} {int(time.time() - t0)}")
    return 1 if failed else 0


def crossmul_main(argv=None):
    """Legacy crossmul: pairs ``slc1 slc2 out`` from ``input_file``, the union
    box of the two headers (crossmul.cu:174-213), zero-filled outside each
    raster; ``found empty image`` for an empty look grid."""
    argv = list(sys.argv if argv is None else argv)
    if len(argv) < 5:
        print(USAGE_CROSSMUL)
        return 0
    _set_gpu(argv)
    input_file, rowlook, collook, out_float = argv[1], int(argv[2]), int(argv[3]), int(argv[4]) != 0
    import torch

    from . import formats
    from .interfere import crossmul_pair
    pairs = []
    with open(input_file) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3:
                pairs.append(parts[:3])
    for a, b, out in pairs:
        h1, d1 = formats.read_raster(a)
        h2, d2 = formats.read_raster(b)
        r = crossmul_pair(h1, torch.from_numpy(d1).cuda(), h2, torch.from_numpy(d2).cuda(), rowlook, collook,
                          out_float=out_float, with_coherence=False, use_union=True)
        if r is None or min(r["phase" if out_float else "ifg"].shape) == 0:
            print("found empty image")
            continue
        print(out)
        formats.write_raster(out, r["header"], (r["phase"] if out_float else r["ifg"]).cpu().numpy())
    return 0


def goldstein_inputs(in_str):
    """A single ``*.int`` file, or the lines of a list file
    (goldstein.cu:55-81); returns (paths, is_single_ifg)."""
    if in_str.endswith(".int"):
        return [in_str], True
    if not os.path.isfile(in_str):
        return [], False
    with open(in_str) as f:
        return [ln.rstrip("\n") for ln in f], False


def goldstein_main(argv=None):
    """Goldstein filter of raw complex64 nrow x ncol images.  Output names as
    goldstein.cu:469-481: ``filtered.int`` for a single ``.int`` input,
    ``<in>.filt`` or ``<in><out_str>`` for list entries.  For a single
    ``.int`` with ``out_str`` the reference leaves its output name empty and
    writes nothing; s1b writes ``<in><out_str>`` there."""
    argv = list(sys.argv if argv is None else argv)
    if len(argv) < 6:
        print(USAGE_GOLDSTEIN)
        return 0
    _set_gpu(argv)
    in_str, nrow, ncol, n_win, alpha = argv[1], int(argv[2]), int(argv[3]), int(argv[4]), float(argv[5])
    out_str = argv[6] if len(argv) > 6 and argv[6] not in ("--gpu", "-g") else ""
    files, single = goldstein_inputs(in_str)
    if not files:
        print("Input list is empty, nothing to filter.")
        return 0
    import torch

    from . import kernels
    scratch = torch.empty(kernels.goldstein_scratch_bytes(nrow, ncol, n_win), dtype=torch.uint8, device="cuda")
    for fin in files:
        if single:
            fout = "filtered.int" if not out_str else fin + out_str
        else:
            fout = fin + (out_str if out_str else ".filt")
        print(f"Run Goldstein filter, input: {fin}, output: {fout}")
        if not os.path.isfile(fin):
            print(f"File {fin} does not exist.")
            data = np.zeros((nrow, ncol), dtype=np.complex64)
        else:
            data = np.fromfile(fin, dtype=np.complex64, count=nrow * ncol)
            if data.size < nrow * ncol:  # the reference reads a short file into a partly stale buffer
                data = np.concatenate([data, np.zeros(nrow * ncol - data.size, np.complex64)])
            data = data.reshape(nrow, ncol)
        out = kernels.goldstein(torch.from_numpy(data).cuda(), alpha, n_win, scratch=scratch)
        out.cpu().numpy().tofile(fout)
    return 0
