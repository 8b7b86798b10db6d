"""The per-burst-pair interferogram chain on one GPU:

    deramp(ref), deramp(sec) -> geo2rdr(ref), geo2rdr(sec) onto the DEM grid
    -> crossmul + multilook + amplitude looks + coherence -> Goldstein

This is what the reference runs as ``geo2rdr`` (twice), ``crossmul_daemon``,
NumPy ``coherence`` and ``goldstein`` with files in between
(s1proc/sentinel_scene.py, interfere.py, coherence.py, phase_correction.py).
Buffers are allocated once per burst geometry and reused, so a step only
launches kernels; the one host synchronisation per pair reads the four crop
rows that size the interferogram (as the reference reads them back before
writing the ``.gslc`` header).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib, formats, kernels, plan as _plan


def _start_event(sink):
    if sink is None:
        return None
    e = torch.cuda.Event(enable_timing=True)
    e.record()
    return e


def _end_event(sink, start):
    if sink is None:
        return
    e = torch.cuda.Event(enable_timing=True)
    e.record()
    sink.append((start, e))


@dataclass
class PairResult:
    header: np.ndarray  # ifg header, int32[64]
    box: tuple          # full-resolution box (left, top, right, bottom)
    ifg: torch.Tensor   # complex64 [nrow_ml, ncol_ml]
    amp1: torch.Tensor
    amp2: torch.Tensor
    coh: torch.Tensor
    filt: torch.Tensor  # Goldstein-filtered ifg
    gslc_headers: tuple


class PairChain:
    """Plans and device buffers for one reference/secondary burst pair."""

    def __init__(self, ref_acq, sec_acq, rsc, rowlook, collook, alpha, n_win=32, device="cuda", burst=0,
                 fill_seed=0):
        self.rowlook, self.collook, self.alpha, self.n_win = int(rowlook), int(collook), float(alpha), int(n_win)
        self.fill_seed = int(fill_seed)
        self.dev = torch.device(device)
        self.plans = [_plan.burst_plan(a.radar, a.orbit, a.fm, a.dc, a.bursts[burst], rsc) for a in (ref_acq, sec_acq)]
        for p in self.plans:
            if p.nrow <= 0 or p.ncol <= 0:
                raise _lib.S1BError(_lib.S1B_ERR_EMPTY, "PairChain: burst outside the DEM grid")
        L, S = self.plans[0].lines, self.plans[0].samples
        self.deramped = [torch.empty(p.lines * p.samples, dtype=torch.complex64, device=self.dev) for p in self.plans]
        self.geo = [torch.empty((p.nrow, p.ncol), dtype=torch.complex64, device=self.dev) for p in self.plans]
        self.rows = torch.empty(4, dtype=torch.int32, device=self.dev)
        self.rows_host = torch.empty(4, dtype=torch.int32, pin_memory=torch.cuda.is_available())
        self.burst_pixels = L * S
        self._scratch = None
        self._ml_shape = None
        self.geo_events = None  # list to collect (start, end) CUDA events around geocoding launches

    def geocode(self, ref_slc: torch.Tensor, sec_slc: torch.Tensor, dem: torch.Tensor):
        for i, (p, slc) in enumerate(zip(self.plans, (ref_slc, sec_slc))):
            kernels.deramp(p, slc.reshape(-1), out=self.deramped[i])
            ev = _start_event(self.geo_events)
            kernels.geo2rdr(p, dem, self.deramped[i], out=self.geo[i], rows=self.rows[2 * i:2 * i + 2])
            _end_event(self.geo_events, ev)

    def headers(self):
        """Crop rows -> the two ``.gslc`` headers (geo2rdr.cu:641-647), or None if a burst is empty."""
        self.rows_host.copy_(self.rows, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        r = self.rows_host.tolist()
        hs = []
        for i, p in enumerate(self.plans):
            first, last = r[2 * i], r[2 * i + 1]
            if first >= p.nrow or last <= first:
                return None
            hs.append(formats.make_header(p.rsc_nlat, p.rsc_nlon, p.win_left, p.win_top + first, p.win_right,
                                          p.win_top + last))
        return hs

    def interfere(self, hs) -> PairResult | None:
        box, hdr6 = _plan.crossmul_box(hs[0], hs[1], self.rowlook, self.collook)
        if box is None:
            return None
        p1, p2 = self.plans
        # the geocoded windows are passed whole: the box lies inside both crops
        outs = kernels.crossmul_looks(self.geo[0], (p1.win_left, p1.win_top), self.geo[1], (p2.win_left, p2.win_top),
                                      box, self.rowlook, self.collook, fill_seed=self.fill_seed)
        ifg = outs["ifg"]
        if ifg.shape[0] >= self.n_win and ifg.shape[1] >= self.n_win:
            if self._ml_shape != tuple(ifg.shape):
                need = kernels.goldstein_scratch_bytes(ifg.shape[0], ifg.shape[1], self.n_win)
                self._scratch = torch.empty(need, dtype=torch.uint8, device=self.dev)
                self._ml_shape = tuple(ifg.shape)
            filt = kernels.goldstein(ifg, self.alpha, self.n_win, scratch=self._scratch)
        else:
            filt = ifg.clone()
        return PairResult(header=formats.make_header(*hdr6), box=tuple(box), ifg=ifg, amp1=outs["amp1"],
                          amp2=outs["amp2"], coh=outs["coh"], filt=filt, gslc_headers=tuple(hs))

    def run(self, ref_slc: torch.Tensor, sec_slc: torch.Tensor, dem: torch.Tensor) -> PairResult | None:
        """One full chain step on device-resident inputs."""
        self.geocode(ref_slc, sec_slc, dem)
        hs = self.headers()
        if hs is None:
            return None
        return self.interfere(hs)

    @staticmethod
    def launches_per_step():
        # 2 x (deramp + rows init + geo2rdr) + crossmul + goldstein (patch + gather)
        return 2 * 3 + 1 + 2


def process_pair_host(chain: PairChain, ref_host: torch.Tensor, sec_host: torch.Tensor, dem_host: torch.Tensor,
                      dev_in=None, host_out=None):
    """End-to-end call on host buffers: H2D of both SLCs and the DEM, the chain,
    D2H of the interferogram, amplitudes, coherence and filtered phase.

    ``dev_in``/``host_out`` are reusable buffers (dicts) so repeated calls do
    not allocate; host tensors should be pinned for asynchronous copies.
    Returns (result, host_out, bytes_h2d, bytes_d2h).
    """
    dev = chain.dev
    if dev_in is None:
        dev_in = {"ref": torch.empty_like(ref_host, device=dev), "sec": torch.empty_like(sec_host, device=dev),
                  "dem": torch.empty_like(dem_host, device=dev)}
    dev_in["ref"].copy_(ref_host, non_blocking=True)
    dev_in["sec"].copy_(sec_host, non_blocking=True)
    dev_in["dem"].copy_(dem_host, non_blocking=True)
    h2d = sum(t.numel() * t.element_size() for t in (ref_host, sec_host, dem_host))
    res = chain.run(dev_in["ref"], dev_in["sec"], dev_in["dem"])
    if res is None:
        return None, host_out, h2d, 0
    outs = {"ifg": res.ifg, "amp1": res.amp1, "amp2": res.amp2, "coh": res.coh, "filt": res.filt}
    if host_out is None or any(host_out[k].shape != v.shape for k, v in outs.items()):
        host_out = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True) for k, v in outs.items()}
    for k, v in outs.items():
        host_out[k].copy_(v, non_blocking=True)
    torch.cuda.current_stream().synchronize()
    d2h = sum(t.numel() * t.element_size() for t in host_out.values())
    return res, host_out, h2d, d2h


class FrameChain:
    """All burst pairs of a frame (subswaths x bursts of uneven size)
    processed pair by pair with shared device buffers sized for the
    largest burst and DEM window."""

    def __init__(self, refs, secs, rsc, rowlook, collook, alpha, n_win=32, device="cuda", fill_seed=0):
        self.dev = torch.device(device)
        self.rowlook, self.collook, self.alpha, self.n_win = int(rowlook), int(collook), float(alpha), int(n_win)
        self.pairs = []
        for ra, sa in zip(refs, secs):
            pls = [_plan.burst_plan(a.radar, a.orbit, a.fm, a.dc, a.bursts[0], rsc) for a in (ra, sa)]
            if any(p.nrow <= 0 or p.ncol <= 0 for p in pls):
                raise _lib.S1BError(_lib.S1B_ERR_EMPTY, "FrameChain: burst outside the DEM grid")
            self.pairs.append(pls)
        max_burst = max(p.lines * p.samples for pls in self.pairs for p in pls)
        max_geo = max(p.nrow * p.ncol for pls in self.pairs for p in pls)
        self.deramped = [torch.empty(max_burst, dtype=torch.complex64, device=self.dev) for _ in range(2)]
        self.geo = [torch.empty(max_geo, dtype=torch.complex64, device=self.dev) for _ in range(2)]
        self.rows = torch.empty(4 * len(self.pairs), dtype=torch.int32, device=self.dev)
        self.rows_host = torch.empty(4 * len(self.pairs), dtype=torch.int32,
                                     pin_memory=torch.cuda.is_available())
        self.burst_pixels = sum(pls[0].lines * pls[0].samples for pls in self.pairs)
        self.fill_seed = int(fill_seed)
        self._scratch = torch.empty(0, dtype=torch.uint8, device=self.dev)
        self.geo_events = None

    def _geo_view(self, i, p):
        return self.geo[i][:p.nrow * p.ncol].view(p.nrow, p.ncol)

    def run_pair(self, k, ref_slc, sec_slc, dem):
        pls = self.pairs[k]
        for i, (p, slc) in enumerate(zip(pls, (ref_slc, sec_slc))):
            kernels.deramp(p, slc.reshape(-1), out=self.deramped[i][:p.lines * p.samples])
            ev = _start_event(self.geo_events)
            kernels.geo2rdr(p, dem, self.deramped[i][:p.lines * p.samples], out=self._geo_view(i, p),
                            rows=self.rows[4 * k + 2 * i:4 * k + 2 * i + 2])
            _end_event(self.geo_events, ev)
        self.rows_host[4 * k:4 * k + 4].copy_(self.rows[4 * k:4 * k + 4], non_blocking=True)
        torch.cuda.current_stream().synchronize()
        r = self.rows_host[4 * k:4 * k + 4].tolist()
        hs = []
        for i, p in enumerate(pls):
            first, last = r[2 * i], r[2 * i + 1]
            if first >= p.nrow or last <= first:
                return None
            hs.append(formats.make_header(p.rsc_nlat, p.rsc_nlon, p.win_left, p.win_top + first, p.win_right,
                                          p.win_top + last))
        box, hdr6 = _plan.crossmul_box(hs[0], hs[1], self.rowlook, self.collook)
        if box is None:
            return None
        p1, p2 = pls
        outs = kernels.crossmul_looks(self._geo_view(0, p1), (p1.win_left, p1.win_top), self._geo_view(1, p2),
                                      (p2.win_left, p2.win_top), box, self.rowlook, self.collook,
                                      fill_seed=self.fill_seed)
        ifg = outs["ifg"]
        filt = ifg
        if ifg.shape[0] >= self.n_win and ifg.shape[1] >= self.n_win:
            need = kernels.goldstein_scratch_bytes(ifg.shape[0], ifg.shape[1], self.n_win)
            if self._scratch.numel() < need:
                self._scratch = torch.empty(need, dtype=torch.uint8, device=self.dev)
            filt = kernels.goldstein(ifg, self.alpha, self.n_win, scratch=self._scratch)
        return PairResult(header=formats.make_header(*hdr6), box=tuple(box), ifg=ifg, amp1=outs["amp1"],
                          amp2=outs["amp2"], coh=outs["coh"], filt=filt, gslc_headers=tuple(hs))

    def run(self, ref_slcs, sec_slcs, dem):
        return [self.run_pair(k, r, s, dem) for k, (r, s) in enumerate(zip(ref_slcs, sec_slcs))]

    def launches_per_step(self):
        return len(self.pairs) * PairChain.launches_per_step()

    def geo_pixels(self):
        return [p.nrow * p.ncol for pls in self.pairs for p in pls]

    def burst_pixels_all(self):
        return [p.lines * p.samples for pls in self.pairs for p in pls]


class RadarChain:
    """Radar-grid chain for one burst pair:
    secondary offsets from the reference grid's float64 lat/lon/height,
    TOPS-aware 8-tap sinc resampling of the secondary onto the reference grid,
    crossmul + multilook + amplitude looks, 5 x 5 full-resolution coherence,
    Goldstein.  No host synchronisation: a step can be captured in a CUDA
    graph (``capture``) and replayed."""

    def __init__(self, ref_acq, sec_acq, lines, samples, rowlook, collook, alpha, win=5, n_win=32,
                 interp="sinc8", device="cuda", fill_seed=0):
        self.dev = torch.device(device)
        self.sec_plan = _plan.burst_plan(sec_acq.radar, sec_acq.orbit, sec_acq.fm, sec_acq.dc, sec_acq.bursts[0],
                                         None)
        self.L, self.S = int(lines), int(samples)
        self.rowlook, self.collook, self.alpha, self.win, self.n_win = (int(rowlook), int(collook), float(alpha),
                                                                        int(win), int(n_win))
        self.interp = interp
        self.fill_seed = int(fill_seed)
        L, S = self.L, self.S
        self.az = torch.empty((L, S), dtype=torch.float32, device=self.dev)
        self.rg = torch.empty((L, S), dtype=torch.float32, device=self.dev)
        self.sec_rs = torch.empty((L, S), dtype=torch.complex64, device=self.dev)
        self.coh_full = torch.empty((L, S), dtype=torch.float32, device=self.dev)
        # staging status words: [0] resample, [1] box coherence (1 = a tile's copy did not complete)
        self.status = torch.zeros(2, dtype=torch.int32, device=self.dev)
        self.box = (0, 0, (S // self.collook) * self.collook, (L // self.rowlook) * self.rowlook)
        nml = (L // self.rowlook, S // self.collook)
        need = kernels.goldstein_scratch_bytes(nml[0], nml[1], self.n_win) if min(nml) >= self.n_win else 0
        self.scratch = torch.empty(max(need, 1), dtype=torch.uint8, device=self.dev)
        self.filt = torch.empty(nml, dtype=torch.complex64, device=self.dev)
        self.burst_pixels = L * S
        self.outs = None
        self.graph = None
        self.geo_events = None

    def run(self, ref_slc, sec_slc, lat, lon, hgt):
        ev = _start_event(self.geo_events)
        kernels.geo2rdr_offsets(self.sec_plan, lat, lon, hgt, self.az, self.rg)
        _end_event(self.geo_events, ev)
        kernels.resample(self.sec_plan, sec_slc, self.az, self.rg, self.interp, out=self.sec_rs,
                         status=self.status[0:1])
        outs = kernels.crossmul_looks(ref_slc, (0, 0), self.sec_rs, (0, 0), self.box, self.rowlook, self.collook,
                                      fill_seed=self.fill_seed)
        kernels.box_coherence(ref_slc, self.sec_rs, self.win, out=self.coh_full, status=self.status[1:2])
        if self.filt.shape[0] >= self.n_win and self.filt.shape[1] >= self.n_win:
            kernels.goldstein(outs["ifg"], self.alpha, self.n_win, out=self.filt, scratch=self.scratch)
        outs["filt"] = self.filt
        outs["coh_full"] = self.coh_full
        self.outs = outs
        return outs

    def capture(self, ref_slc, sec_slc, lat, lon, hgt):
        """Record one step into a CUDA graph on static inputs; ``replay()`` reruns it."""
        self.run(ref_slc, sec_slc, lat, lon, hgt)  # warm-up outside the capture (attributes, scratch)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run(ref_slc, sec_slc, lat, lon, hgt)
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g
        return self.outs

    def replay(self):
        self.graph.replay()
        return self.outs

    def staging_ok(self) -> bool:
        """True when no tile of the last step lost a shared-memory copy (synchronises)."""
        return not bool(self.status.any().item())

    @staticmethod
    def launches_per_step():
        # offsets, resample, crossmul, box coherence (+ status memset), goldstein patch + gather
        return 6


FRAME_LIST_MAX = 240  # bursts per deramp launch (kFrameListMax, csrc/s1b_frame.h)


TUNING_FIELDS = ("deramp_rows", "deramp_ctas", "geo_cols", "geo_ctas")


def tuning_cache_path():
    """The frame autotuner's cache file: ``$S1B_TUNING_CACHE``, else
    ``$XDG_CACHE_HOME/s1b/frame_tuning.json`` (``~/.cache`` by default)."""
    import os
    p = os.environ.get("S1B_TUNING_CACHE")
    if p:
        return p
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "s1b", "frame_tuning.json")


def tuning_key(gpu_name, capability, sm_count, sample_format, deramp_fused, crossmul_fused, bursts):
    """Key of a frame's shape class on one kind of GPU: the GPU (name,
    compute capability, SM count), the frame's stage forms and its bursts'
    count and median size, lines to 256 and samples to 2048 (the tile choices
    depend on the burst shapes and the SM count, not on exact sizes)."""
    lines = sorted(int(b[0]) for b in bursts)
    samples = sorted(int(b[1]) for b in bursts)
    ml, ms = lines[len(lines) // 2], samples[len(samples) // 2]
    shape = f"{len(bursts)}x{(ml + 128) // 256 * 256}x{(ms + 1024) // 2048 * 2048}"
    return (f"{gpu_name}|cc{capability[0]}.{capability[1]}|sm{sm_count}|{sample_format}|"
            f"deramp={'fused' if deramp_fused else 'kernel'}|crossmul={'fused' if crossmul_fused else 'kernel'}|{shape}")


def load_tuning(path):
    """The cache's entries ({key: tuning dict}); empty when the file is
    missing or unreadable, and entries without the four fields are dropped."""
    import json
    try:
        with open(path) as f:
            d = json.load(f)
    except (OSError, ValueError):
        return {}
    if not isinstance(d, dict):
        return {}
    return {k: {f: int(v[f]) for f in TUNING_FIELDS} for k, v in d.items()
            if isinstance(v, dict) and all(isinstance(v.get(f), int) for f in TUNING_FIELDS)}


def store_tuning(path, key, tuning):
    """Add or replace one entry; the file is replaced atomically, so
    concurrent writers (ranks on one node) leave a complete file."""
    import json
    import os
    import tempfile
    d = load_tuning(path)
    d[key] = {f: int(tuning[f]) for f in TUNING_FIELDS}
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    fd, tmp = tempfile.mkstemp(dir=os.path.dirname(os.path.abspath(path)), suffix=".tmp")
    with os.fdopen(fd, "w") as f:
        json.dump(d, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


class BatchedFrameChain:
    """All burst pairs of a frame through one batched launch sequence
    (``s1b_frame_run``): deramp and geocoding over every burst (one CTA per
    tile, or persistent grids; the autotuner picks), the crossmul box of each pair formed on the device, crossmul and
    Goldstein over all pairs.  No host synchronisation inside a run, so it is
    captured in a CUDA graph (``capture``/``replay``).  Per-pair products are
    those of :class:`FrameChain` (same kernels, same order of operations).

    The SLCs live back to back in one device buffer; ``ref_views``/``sec_views``
    are the per-burst views to fill.  ``sample_format="ci16"`` keeps them as
    the measurement TIFF's complex int16 samples (int16 [lines, samples, 2],
    half the bytes to move and to read), widened where they are read; the
    products equal those of the complex64 buffer holding the same values.
    ``deramp_fused`` (default): the geocoding deramps the samples of each
    bilinear gather itself (no deramped copy of the bursts); False runs a
    deramp kernel first.  The products agree to float rounding.
    ``crossmul_fused`` (default): the geocoding kernel geocodes both bursts
    of a pair at each DEM pixel and forms the crossmul's look-row sums (no
    geocoded windows are written); False geocodes every window and runs the
    crossmul kernel on them.  The products agree to float rounding.
    ``autotune`` picks the deramp and geocoding tile shapes and grid sizes on
    the actual frame.
    """

    def __init__(self, refs, secs, rsc, rowlook, collook, alpha, n_win=32, device="cuda", fill_seed=0,
                 sample_format="c64", deramp_fused=True, crossmul_fused=True, pairs=None):
        import ctypes
        if sample_format not in ("c64", "ci16"):
            raise ValueError("sample_format must be 'c64' (complex64) or 'ci16' (complex int16)")
        self.sample_format = sample_format
        self.dev = torch.device(device)
        self.rowlook, self.collook, self.alpha, self.n_win = int(rowlook), int(collook), float(alpha), int(n_win)
        self.fill_seed = int(fill_seed)
        if pairs is None:
            # refs[k] with secs[k]: bursts 2k and 2k + 1
            acqs = [a for ra, sa in zip(refs, secs) for a in (ra, sa)]
            pairs = [(2 * k, 2 * k + 1) for k in range(len(refs))]
        else:
            # ``refs`` lists every burst once; ``pairs`` indexes into it (a
            # burst shared by several pairs, e.g. a stack's reference date, is
            # stored and geocoded once when the crossmul is not fused)
            acqs = list(refs)
            pairs = [(int(a), int(b)) for a, b in pairs]
            if any(not (0 <= i < len(acqs)) for pr in pairs for i in pr):
                raise ValueError("pair index outside the burst list")
        plans = []
        for a in acqs:
            p = _plan.burst_plan(a.radar, a.orbit, a.fm, a.dc, a.bursts[0], rsc)
            if p.nrow <= 0 or p.ncol <= 0:
                raise _lib.S1BError(_lib.S1B_ERR_EMPTY, "BatchedFrameChain: burst outside the DEM grid")
            plans.append(p)
        self.plans = plans
        self.pair_index = pairs
        self.n_pairs = len(pairs)
        lib = _lib.load()
        arr = (_lib.BurstPlan * len(plans))(*plans)
        pref = (ctypes.c_int32 * self.n_pairs)(*[a for a, _ in pairs])
        psec = (ctypes.c_int32 * self.n_pairs)(*[b for _, b in pairs])
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.dev):
            _lib.check(lib.s1b_frame_create(arr, len(plans), pref, psec, self.n_pairs, self.rowlook, self.collook,
                                            self.n_win, self.alpha, self.fill_seed, ctypes.byref(handle)),
                       "s1b_frame_create")
        self._handle = handle
        if sample_format == "ci16":
            _lib.check(lib.s1b_frame_set_sample_format(handle, _lib.S1B_SAMPLES_CI16), "s1b_frame_set_sample_format")
        self.deramp_fused = bool(deramp_fused)
        _lib.check(lib.s1b_frame_set_deramp_fusion(handle, int(self.deramp_fused)), "s1b_frame_set_deramp_fusion")
        self.crossmul_fused = bool(crossmul_fused) and self.rowlook <= 128
        _lib.check(lib.s1b_frame_set_crossmul_fusion(handle, int(self.crossmul_fused)),
                   "s1b_frame_set_crossmul_fusion")
        sz = _lib.FrameSizes()
        _lib.check(lib.s1b_frame_sizes(handle, ctypes.byref(sz)), "s1b_frame_sizes")
        self.sizes = sz
        if sample_format == "ci16":
            self.slc = torch.empty((int(sz.slc_elems), 2), dtype=torch.int16, device=self.dev)
        else:
            self.slc = torch.empty(int(sz.slc_elems), dtype=torch.complex64, device=self.dev)
        self.workspace = torch.empty(int(sz.workspace_bytes), dtype=torch.uint8, device=self.dev)
        n = int(sz.product_elems)
        self.ifg = torch.empty(n, dtype=torch.complex64, device=self.dev)
        self.filt = torch.empty(n, dtype=torch.complex64, device=self.dev)
        self.amp1 = torch.empty(n, dtype=torch.float32, device=self.dev)
        self.amp2 = torch.empty(n, dtype=torch.float32, device=self.dev)
        self.coh = torch.empty(n, dtype=torch.float32, device=self.dev)
        self.pair_size = ctypes.sizeof(_lib.FramePair)
        self.pairs_dev = torch.zeros(self.n_pairs * self.pair_size, dtype=torch.uint8, device=self.dev)
        self.pairs_host = torch.empty(self.n_pairs * self.pair_size, dtype=torch.uint8,
                                      pin_memory=torch.cuda.is_available())
        views, self.burst_offsets = [], []
        for b, p in enumerate(plans):
            off = ctypes.c_int64()
            _lib.check(lib.s1b_frame_burst_offset(handle, b, ctypes.byref(off)), "s1b_frame_burst_offset")
            self.burst_offsets.append(off.value)
            v = self.slc[off.value:off.value + p.lines * p.samples]
            views.append(v.view(p.lines, p.samples, 2) if sample_format == "ci16" else v.view(p.lines, p.samples))
        self.views = views
        self.ref_views = [views[a] for a, _ in pairs]
        self.sec_views = [views[b] for _, b in pairs]
        self.slots = []
        for k in range(self.n_pairs):
            off, r, c = ctypes.c_int64(), ctypes.c_int32(), ctypes.c_int32()
            _lib.check(lib.s1b_frame_pair_slot(handle, k, ctypes.byref(off), ctypes.byref(r), ctypes.byref(c)),
                       "s1b_frame_pair_slot")
            self.slots.append((off.value, r.value, c.value))
        self.burst_pixels = sum(plans[a].lines * plans[a].samples for a, _ in pairs)
        self.tuning_source = "default"  # "timed" or "cache" once autotuned
        self.graph = None
        self.geo_events = None

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().s1b_frame_destroy(h)
            except Exception:
                pass
            self._handle = None

    def _args(self, dem, slc=None):
        if dem.dtype != torch.int16 or dem.dim() != 2 or dem.stride(1) != 1 or dem.device != self.dev:
            raise ValueError("dem must be an int16 [nlat, nlon] device raster with unit column stride")
        if dem.shape[0] < max(p.win_bottom for p in self.plans) or dem.shape[1] < max(p.win_right for p in self.plans):
            raise ValueError("dem does not cover every burst's DEM window")
        slc = self.slc if slc is None else slc
        if slc.dtype != self.slc.dtype or slc.shape != self.slc.shape or not slc.is_contiguous() or slc.device != self.dev:
            raise ValueError("slc must be a contiguous buffer like chain.slc")
        return (self._handle, _lib.dptr(slc), _lib.dptr(dem), dem.stride(0), _lib.dptr(self.workspace),
                _lib.dptr(self.ifg), _lib.dptr(self.amp1), _lib.dptr(self.amp2), _lib.dptr(self.coh),
                _lib.dptr(self.filt), _lib.dptr(self.pairs_dev))

    def load(self, ref_slcs, sec_slcs):
        """Copy per-burst SLCs (device or pinned host tensors) into the frame buffer."""
        for v, s in zip(self.ref_views + self.sec_views, list(ref_slcs) + list(sec_slcs)):
            v.copy_(s.reshape(v.shape), non_blocking=True)

    def run(self, dem, slc=None):
        """One frame run on the current stream (inputs already in ``slc``,
        default the chain's own buffer; another buffer must have its layout,
        e.g. ``torch.empty_like(chain.slc)``)."""
        _lib.check(_call_frame("frame_run", _lib.load().s1b_frame_run, *self._args(dem, slc), _lib.stream_ptr()),
                   "s1b_frame_run")

    def autotune(self, dem, reps=3, cache=True):
        """Time the tile-shape / grid candidates on this frame and keep the
        fastest.  With ``cache``, the choice is kept in the tuning cache
        (``tuning_cache_path``) under this GPU and the frame's shape class
        (``tuning_key``), and a later frame of that class on that GPU takes it
        from there without timing anything."""
        key = path = None
        if cache:
            props = torch.cuda.get_device_properties(self.dev)
            key = tuning_key(props.name, (props.major, props.minor), props.multi_processor_count,
                             self.sample_format, self.deramp_fused, self.crossmul_fused,
                             [(p.lines, p.samples) for p in self.plans])
            path = tuning_cache_path()
            hit = load_tuning(path).get(key)
            if hit is not None:
                self.set_tuning(**hit)
                self.tuning_source = "cache"
                return self.tuning()
        _lib.check(_lib.load().s1b_frame_autotune(*self._args(dem), int(reps), _lib.stream_ptr()),
                   "s1b_frame_autotune")
        self.tuning_source = "timed"
        t = self.tuning()
        if cache:
            store_tuning(path, key, t)
        return t

    def profile(self, dem):
        """One run with CUDA events between stages: ms of deramp, geocoding, box,
        crossmul, Goldstein (synchronises)."""
        import ctypes
        ms = (ctypes.c_float * 5)()
        _lib.check(_lib.load().s1b_frame_profile(*self._args(dem), ms, _lib.stream_ptr()), "s1b_frame_profile")
        return dict(zip(("deramp", "geo2rdr", "box", "crossmul_looks", "goldstein"), list(ms)))

    def tuning(self):
        import ctypes
        t = (ctypes.c_int32 * 4)()
        _lib.check(_lib.load().s1b_frame_tuning(self._handle, t), "s1b_frame_tuning")
        return {"deramp_rows": t[0], "deramp_ctas": t[1], "geo_cols": t[2], "geo_ctas": t[3]}

    def set_tuning(self, deramp_rows=16, deramp_ctas=0, geo_cols=128, geo_ctas=0):
        import ctypes
        t = (ctypes.c_int32 * 4)(deramp_rows, deramp_ctas, geo_cols, geo_ctas)
        _lib.check(_lib.load().s1b_frame_set_tuning(self._handle, t), "s1b_frame_set_tuning")

    def capture(self, dem, slc=None):
        """Record one frame run into a CUDA graph; ``replay()`` reruns it.
        With ``slc`` (another buffer like ``chain.slc``) the graph is returned
        instead of kept as the chain's."""
        self.run(dem, slc)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                self.run(dem, slc)
        torch.cuda.current_stream().wait_stream(s)
        if slc is not None:
            return g
        self.graph = g
        return g

    def replay(self):
        self.graph.replay()

    def pair_table(self):
        """Per-pair results of the last run (synchronises): list of dicts."""
        import ctypes
        self.pairs_host.copy_(self.pairs_dev, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        raw = bytes(self.pairs_host.numpy())
        out = []
        for k in range(self.n_pairs):
            r = _lib.FramePair.from_buffer_copy(raw[k * self.pair_size:(k + 1) * self.pair_size])
            out.append({"ok": bool(r.ok), "nrow_ml": r.nrow_ml, "ncol_ml": r.ncol_ml, "filtered": bool(r.filtered),
                        "header": list(r.header), "box": tuple(r.box), "gslc_rows": list(r.gslc_rows)})
        return out

    def results(self):
        """PairResult per pair (views into the product arrays), None for empty pairs."""
        res = []
        for k, r in enumerate(self.pair_table()):
            if not r["ok"]:
                res.append(None)
                continue
            off = self.slots[k][0]
            n = r["nrow_ml"] * r["ncol_ml"]
            shape = (r["nrow_ml"], r["ncol_ml"])
            p1, p2 = self.plans[self.pair_index[k][0]], self.plans[self.pair_index[k][1]]
            g = r["gslc_rows"]
            hs = (formats.make_header(p1.rsc_nlat, p1.rsc_nlon, p1.win_left, p1.win_top + g[0], p1.win_right,
                                      p1.win_top + g[1]),
                  formats.make_header(p2.rsc_nlat, p2.rsc_nlon, p2.win_left, p2.win_top + g[2], p2.win_right,
                                      p2.win_top + g[3]))
            res.append(PairResult(header=formats.make_header(*r["header"]), box=r["box"],
                                  ifg=self.ifg[off:off + n].view(shape), amp1=self.amp1[off:off + n].view(shape),
                                  amp2=self.amp2[off:off + n].view(shape), coh=self.coh[off:off + n].view(shape),
                                  filt=self.filt[off:off + n].view(shape), gslc_headers=hs))
        return res

    def launches_per_step(self):
        """Kernels one run launches: init, geocoding, box, crossmul, Goldstein
        patches and gather, plus the deramp: one persistent launch, or one
        CTA-per-tile launch per load width (16-byte rows or not) and per list
        of up to FRAME_LIST_MAX bursts."""
        t = self.tuning()
        if self.deramp_fused or t["deramp_ctas"]:  # column tables, or one persistent deramp
            return 7
        base = self.slc.data_ptr()
        es = 4 if self.sample_format == "ci16" else 8
        vec = sum(1 for p, off in zip(self.plans, self.burst_offsets)
                  if p.samples % 2 == 0 and (base + es * off) % (2 * es) == 0)
        per = FRAME_LIST_MAX
        return 6 + -(-vec // per) + -(-(len(self.plans) - vec) // per)

    def geo_pixels(self):
        return [p.nrow * p.ncol for p in self.plans]

    def burst_pixels_all(self):
        return [p.lines * p.samples for p in self.plans]


class FramePipeline:
    """Frames streamed through one ``BatchedFrameChain`` with host buffers.

    Two input slots (SLC buffer and DEM) alternate, each with its own CUDA
    graph of the frame run: ``submit`` enqueues the host-to-device copy of a
    frame's bursts (and DEM) on a copy stream, into the slot the frame before
    last used once that frame's run is done, and, on the current stream, the
    run and the device-to-host copy of the products.  So the copy of frame k + 1 crosses PCIe while frame k runs;
    the frames' runs and product reads stay in order on one stream.  Nothing
    synchronises the host: ``host_out`` holds frame k's products once the
    current stream has passed its ``submit``.
    """

    def __init__(self, chain: BatchedFrameChain, dem):
        self.chain = chain
        self.slcs = [chain.slc, torch.empty_like(chain.slc)]
        self.dems = [dem, dem.clone()]
        self.views = []
        for buf in self.slcs:
            vs = []
            for p, off in zip(chain.plans, chain.burst_offsets):
                v = buf[off:off + p.lines * p.samples]
                vs.append(v.view(p.lines, p.samples, 2) if chain.sample_format == "ci16" else v.view(p.lines, p.samples))
            self.views.append(vs[0::2] + vs[1::2])  # the order of chain.ref_views + chain.sec_views
        if chain.graph is None:
            chain.capture(dem)
        self.slcs[1].copy_(self.slcs[0])
        self.graphs = [chain.graph, chain.capture(self.dems[1], self.slcs[1])]
        self.copy = torch.cuda.Stream(chain.dev)
        self.loaded = [torch.cuda.Event() for _ in range(2)]
        self.done = [torch.cuda.Event() for _ in range(2)]
        self.k = 0

    def outputs(self):
        return (self.chain.ifg, self.chain.amp1, self.chain.amp2, self.chain.coh, self.chain.filt)

    def submit(self, host_bursts, host_dem=None, host_out=None):
        """One frame: ``host_bursts`` are its bursts (reference then secondary
        order of ``chain.ref_views + chain.sec_views``), ideally pinned;
        ``host_dem`` its DEM (None: the slot keeps the one it has);
        ``host_out`` optional pinned tensors like ``outputs()``."""
        b = self.k & 1
        cur = torch.cuda.current_stream(self.chain.dev)
        if self.k >= 2:
            self.copy.wait_event(self.done[b])  # the run that read this slot is over
        with torch.cuda.stream(self.copy):
            if host_dem is not None:
                self.dems[b].copy_(host_dem, non_blocking=True)
            for v, h in zip(self.views[b], host_bursts):
                v.copy_(h.reshape(v.shape), non_blocking=True)
            self.loaded[b].record(self.copy)
        cur.wait_event(self.loaded[b])
        self.graphs[b].replay()
        if host_out is not None:
            for h, o in zip(host_out, self.outputs()):
                h.copy_(o, non_blocking=True)
        self.done[b].record(cur)
        self.k += 1


def _call_frame(name, fn, *args):
    return kernels._call(name, fn, *args)
