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
