"""Generate tests/golden/s1proc_pins.npz: outputs of the reference's own Python
for amplitude looks, coherence and burst stitching, on seeded inputs.

The functions run are the reference's, imported from its source tree:
  * s1proc/sario.py:397-420       cpxlooks, powlooks
  * s1proc/coherence.py:14-55     multilook (.gslc files -> .amp mosaic)
  * s1proc/coherence.py:109-147   coherence (.int + .amp -> .cc)
  * s1proc/interfere.py:81-180    stitch_subswath, stitch (burst .int files -> frame)

``s1proc.sario`` imports zarr, matplotlib and numcodecs at module level
(sario.py:8-13) for functions off this path; they are absent here, so empty
stand-in modules are installed in ``sys.modules`` before the import.  None of
the functions above touches them.  The reference fills coherence values
above 1 with unseeded ``np.random.rand`` (coherence.py:142-144); the global
NumPy generator is seeded before the call and the fill mask is stored, so the
tests compare the other pixels exactly and check only the range of the fill.

Usage: ``python tests/golden/make_s1proc_golden.py [--reference DIR]`` (the
reference source tree; default: the one oracle/build_ref.py resolves).
"""
from __future__ import annotations

import argparse
import os
import shutil
import sys
import tempfile
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "s1proc_pins.npz")
NHEAD = 64


def import_reference(reference):
    """Import s1proc.sario, s1proc.coherence and s1proc.interfere from the
    reference source tree, with stand-ins for its off-path imports."""
    for name in ("zarr", "numcodecs", "matplotlib", "matplotlib.pyplot", "matplotlib.colors"):
        if name not in sys.modules:
            sys.modules[name] = types.ModuleType(name)
    class _Unused:  # stands in for off-path classes built at import time (a colour map)
        def __init__(self, *args, **kwargs):
            pass

    sys.modules["numcodecs"].Blosc = _Unused
    sys.modules["matplotlib.colors"].ListedColormap = _Unused
    sys.modules["matplotlib"].pyplot = sys.modules["matplotlib.pyplot"]
    sys.modules["matplotlib"].colors = sys.modules["matplotlib.colors"]
    if reference not in sys.path:
        sys.path.insert(0, reference)
    import s1proc.coherence as coh
    import s1proc.interfere as itf
    import s1proc.sario as sario
    return sario, coh, itf


def write_cropped(path, header6, data):
    h = np.zeros(NHEAD, dtype=np.int32)
    h[:6] = header6
    with open(path, "wb") as f:
        h.tofile(f)
        np.ascontiguousarray(data).tofile(f)


def _speckle(rng, shape, zero_frac=0.0):
    z = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    if zero_frac:
        z[rng.random(shape) < zero_frac] = 0
    return z


def looks_cases(sario, rng, out):
    """cpxlooks / powlooks on complex64 and float32 inputs, several look counts."""
    cases = [((37, 61), 1, 1), ((37, 61), 2, 4), ((40, 160), 4, 20), ((33, 50), 3, 1), ((33, 50), 1, 5)]
    for k, (shape, rl, cl) in enumerate(cases):
        z = _speckle(rng, shape, 0.1)
        out[f"looks{k}_in"] = z
        out[f"looks{k}_rc"] = np.array([rl, cl])
        out[f"looks{k}_cpx"] = sario.cpxlooks(z, rl, cl)
        out[f"looks{k}_pow"] = sario.powlooks(z, rl, cl)


def multilook_case(coh, rng, wd, out):
    """One date's geocoded bursts (.gslc) -> .amp mosaic, first burst whole,
    later ones where it is still 0; crops not aligned to the looks."""
    nrow0, ncol0 = 96, 160
    boxes = [(10, 5, 151, 47), (13, 38, 147, 81), (0, 71, 160, 96)]  # left, top, right, bottom
    files = []
    for i, (l, t, r, b) in enumerate(boxes):
        z = _speckle(rng, (b - t, r - l))
        z[:, :3] = 0  # zero-filled borders, as geocoded windows have
        z[-2:, :] = 0
        f = os.path.join(wd, f"20200101_S1A_AAAA_iw1_burst_{i}.gslc")
        write_cropped(f, [nrow0, ncol0, l, t, r, b], z)
        files.append(f)
        out[f"ml_burst{i}_hdr"] = np.array([nrow0, ncol0, l, t, r, b], dtype=np.int32)
        out[f"ml_burst{i}_data"] = z
    for rl, cl in ((2, 4), (1, 1), (3, 8)):
        amp = os.path.join(wd, f"amp_{rl}x{cl}.amp")
        coh.multilook(files, amp, rl, cl)
        out[f"ml_{rl}x{cl}_amp"] = np.fromfile(amp, dtype=np.float32).reshape(nrow0 // rl, ncol0 // cl)


def coherence_case(coh, rng, wd, out):
    """.int + the two dates' .amp -> .cc rows [amp1 amp2 | coherence]."""
    nrow, ncol = 48, 40
    ifg_dir = os.path.join(wd, "ifg")
    amp_dir = os.path.join(wd, "amp")
    os.makedirs(ifg_dir)
    os.makedirs(amp_dir)
    a1 = (0.5 + rng.random((nrow, ncol))).astype(np.float32)
    a2 = (0.5 + rng.random((nrow, ncol))).astype(np.float32)
    g = rng.random((nrow, ncol)) * 0.95
    g[rng.random((nrow, ncol)) < 0.05] = 1.5  # coherence above 1: the reference's random fill
    ifg = (g * a1 * a2 * np.exp(1j * rng.uniform(-np.pi, np.pi, (nrow, ncol)))).astype(np.complex64)
    ifg[:3, :] = 0
    a1[:3, :5] = 0
    a1.tofile(os.path.join(amp_dir, "20200101.amp"))
    a2.tofile(os.path.join(amp_dir, "20200113.amp"))
    ifg.tofile(os.path.join(ifg_dir, "20200101_20200113.int"))
    np.random.seed(20261203)
    coh.coherence(ifg_dir, amp_dir, nrow, ncol, 2, 4)
    cc = np.fromfile(os.path.join(ifg_dir, "20200101_20200113.cc"), dtype=np.float32).reshape(nrow, 2 * ncol)
    c = np.abs(ifg) / (a1 + np.float32(1e-12)) / (a2 + np.float32(1e-12))
    out.update(coh_ifg=ifg, coh_amp1=a1, coh_amp2=a2, coh_cc=cc, coh_fill=(c > 1))


def stitch_case(itf, rng, wd, out):
    """Burst interferograms of two subswaths -> one frame; the bursts come from
    two products, so the overlap phase offset is estimated where the product
    ids change (interfere.py:92-130)."""
    nrow0, ncol0 = 120, 200
    yy, xx = np.mgrid[0:nrow0, 0:ncol0]
    field = np.exp(1j * (0.05 * xx + 0.03 * yy)).astype(np.complex64)
    # (subswath, product of the reference burst, product of the secondary burst, box, phase offset)
    # middle bursts lie inside the union of the first and last (the subswath
    # bounds, sario.py:230-237), as the bursts of one subswath do
    bursts = [(1, "AAAA", "CCCC", (5, 2, 100, 44), 0.0), (1, "AAAA", "CCCC", (6, 36, 99, 80), 0.0),
              (1, "BBBB", "CCCC", (4, 73, 101, 118), 0.7), (2, "AAAA", "CCCC", (92, 0, 195, 41), -0.4),
              (2, "BBBB", "DDDD", (93, 35, 194, 79), 0.9), (2, "BBBB", "DDDD", (90, 72, 198, 117), 0.9)]
    src = os.path.join(wd, "stitch_src")
    os.makedirs(src)
    names = []
    for k, (sw, p1, p2, (l, t, r, b), off) in enumerate(bursts):
        d = field[t:b, l:r] * np.complex64(np.exp(1j * off))
        d = (d + 0.2 * _speckle(rng, d.shape)).astype(np.complex64)
        d[:, :2] = 0
        d[rng.random(d.shape) < 0.02] = 0
        name = f"20200101_S1A_{p1}_iw{sw}_burst_{k}_20200113_S1A_{p2}_iw{sw}_burst_{k}.int"
        write_cropped(os.path.join(src, name), [nrow0, ncol0, l, t, r, b], d)
        names.append(name)
        out[f"st_burst{k}_hdr"] = np.array([nrow0, ncol0, l, t, r, b], dtype=np.int32)
        out[f"st_burst{k}_data"] = d
        out[f"st_burst{k}_meta"] = np.array([sw, k], dtype=np.int32)
    out["st_names"] = np.array(names)
    run = os.path.join(wd, "stitch_run")
    shutil.copytree(src, run)  # stitch_subswath removes its burst files
    frame = os.path.join(wd, "frame.int")
    itf.stitch([os.path.join(run, n) for n in names], frame, False)
    out["st_frame"] = np.fromfile(frame, dtype=np.complex64).reshape(nrow0, ncol0)
    out["st_shape"] = np.array([nrow0, ncol0])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=None)
    a = ap.parse_args()
    sys.path.insert(0, ROOT)
    from oracle import build_ref
    reference = build_ref.reference_dir(a.reference)
    sario, coh, itf = import_reference(reference)
    rng = np.random.default_rng(20261203)
    out = {}
    wd = tempfile.mkdtemp(prefix="s1proc_golden_")
    try:
        looks_cases(sario, rng, out)
        multilook_case(coh, rng, wd, out)
        coherence_case(coh, rng, wd, out)
        stitch_case(itf, rng, wd, out)
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    main()
