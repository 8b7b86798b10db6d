"""Benchmark: IW-burst pixels/s of the chain geo2rdr -> resample -> ifg -> coherence -> Goldstein.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl s1b|reference] [--config frame|c1]

A step is one pass of the chain over a full synthetic IW frame (default:
3 subswaths x 9 bursts of uneven size, lines 1480-1530, samples
20000-25500, complex64, looks 4 x 20, Goldstein alpha 0.5, 32 x 32 patches)
or over one IW burst pair (--config c1: 1500 x 21000, alpha 0.6):
for every burst pair, TOPS deramp and FP64 geocoding of both SLCs onto the
DEM grid, crossmul + multilook + amplitude looks + coherence, Goldstein.
``value`` = burst pixels (lines x samples of each reference burst, counted
once per pair) per second with inputs resident in HBM; ``e2e`` = the same
with pinned H2D of every SLC and the DEM and D2H of the products inside the
timed region.

With N > 1 (torchrun) every rank processes its own seeded burst pair (weak
scaling, no data-path collective); timings are the max over ranks.

``--impl reference`` times the reference's own implementation on the same
workload: its CUDA executables (built from the reference sources into
oracle/_ref) for geo2rdr x 2, crossmul_daemon and goldstein, and its NumPy
coherence formulas, with the inputs in its file formats on /dev/shm.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "IW-burst px/s (geo2rdr->resample->ifg->coh->Goldstein)"
UNIT = "burst-px/s"
# Algorithmic bytes of the geocoding kernel per launch: DEM window (int16) and
# output (complex64) per geo pixel, the deramped burst read once.
GEO_BYTES_PER_GEO_PX = 2 + 8
GEO_BYTES_PER_BURST_PX = 8
# Measured DRAM traffic (ncu dram__bytes_read.sum + dram__bytes_write.sum of
# one launch on the 1500 x 21000 burst pair, divided by the units it
# processed): geocoding per geo pixel (16.06 M geo px: 285.6 + 93.9 MB) and
# the TMA resampler per output pixel (31.5 M px: 550.9 + 228.7 MB).  Both
# kernels stream their inputs once, so traffic scales with the unit count.
GEO_DRAM_BYTES_PER_GEO_PX = 23.63
# fused frame geocoding (deramp in the gathers): ncu DRAM traffic over algorithmic
# bytes of one launch on the small frame (586.5 MB / 496.1 MB); both terms (raw
# samples read, geocoded pixels written) scale with the frame
GEO_FUSED_TRAFFIC_RATIO = 1.182
# the same with the crossmul look sums formed in the geocoding, per sample format:
# complex64 samples 450.7 MB / 491.7 MB (the gathers touch only the samples the
# DEM window maps into, less than every sample of both bursts), complex int16
# samples 391.7 MB / 290.7 MB
GEO_XMUL_TRAFFIC_RATIO = {"c64": 0.917, "ci16": 1.347}
RESAMPLE_DRAM_BYTES_PER_PX = 24.75
# what bounds the frame geocoding, from its ncu counters (issue and warp stalls)
GEO_LIMITER = ("latency: per-pixel chain of FP64 solve, gathers and phasors at 20 resident warps per SM "
               "(issue active 45 %, XU pipe 30 %, FP64 pipe 22 %); not HBM, not FP64 throughput")
# FP64 operations of the frame geocoding per geocoded DEM pixel (both bursts):
# ncu per-opcode thread-instruction counts of one launch on the small frame
# (29.40 M geocoded pixels): 2 x 581.7 M DFMA + 273.7 M DMUL + 270.6 M DADD.
# Counted before the seed's column term and the line-0 times were hoisted out
# of the pixel loop (up to 15 fewer per pixel since): an upper bound.
GEO_FP64_FLOP_PER_GEO_PX = 58.09


def fp64_peak_tflops(dev):
    """Measured FP64 throughput of this GPU: torch float64 matmul (cuBLAS
    DGEMM) of 4096^3, best of 5, CUDA events."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="s1b", choices=["s1b", "reference"])
    ap.add_argument("--config", default="frame",
                    choices=["frame", "frame_small", "frame_pairs", "c1", "c1geo", "c0", "small", "adjoint", "stack"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the checker leg (pair 0 against the reference executables and the float64 oracle)")
    ap.add_argument("--no-extras", action="store_true",
                    help="frame: skip the extra measurements (complex int16 variant, radar-grid kernels, adjoint)")
    ap.add_argument("--deramp", default="fused", choices=["fused", "kernel"],
                    help="frame deramp: inside the geocoding's gathers, or a separate kernel writing deramped bursts")
    ap.add_argument("--crossmul", default="fused", choices=["fused", "kernel"],
                    help="frame: crossmul look sums formed in the geocoding (fused) or a crossmul kernel reading "
                         "geocoded windows")
    ap.add_argument("--samples", default="c64", choices=["ci16", "c64"],
                    help="frame SLC sample type: complex int16 as in the measurement TIFF (widened on the GPU), "
                         "or complex64 as the reference's geo2rdr pipe carries it")
    ap.add_argument("--adjoint-bursts", type=int, default=8,
                    help="--config adjoint: bursts of 1500 x 21000 (8 as configured; fewer for a profile)")
    ap.add_argument("--write-pair0", metavar="DIR", default=None,
                    help="write burst pair 0 of the frame's SLCs (ref.npy, sec.npy) to DIR and exit: the "
                         "reference arm's inputs, made in a process of their own")
    return ap.parse_args()


def dist_setup(n):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def max_over_ranks(x, world):
    """The slowest rank's value (elapsed times are max-reduced across ranks);
    the tensor lives where the process group's backend reduces (NCCL: the
    GPU, gloo: the host)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world, steps, units_per_step, elapsed_ms):
    """Whole-job throughput of weakly scaled replicas: every rank processes
    ``units_per_step`` per step, the job takes the slowest rank's time."""
    return world * steps * units_per_step / (elapsed_ms / 1e3)


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class Clocks:
    """SM clock and throttle-reason samples during the timed region.

    A background thread polls NVML every 5 ms (the timed region can be far
    shorter than nvidia-smi's 200 ms minimum period); without NVML it falls
    back to ``nvidia-smi -lms 200``.
    """

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, index):
        self.index = index
        self.samples = []
        self.reasons = set()
        self.max_mhz = None
        self._stop = None
        self._thread = None
        self._smi = None

    def start(self):
        import threading
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
        except Exception:  # noqa: BLE001 -- any NVML failure: fall back
            self._start_smi()
            return
        self._stop = threading.Event()

        def loop():
            while not self._stop.is_set():
                try:
                    self.samples.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    for nm, bit in self.REASONS.items():
                        if r & bit:
                            self.reasons.add(nm)
                except Exception:  # noqa: BLE001
                    pass
                self._stop.wait(0.005)

        self._thread = threading.Thread(target=loop, daemon=True)
        self._thread.start()

    def _start_smi(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self._smi = (subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-i",
                                       str(self.index), "-lms", "200"], stdout=open(path, "w"),
                                      stderr=subprocess.DEVNULL), path)

    def stop(self):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=2)
        elif self._smi is not None:
            proc, path = self._smi
            proc.terminate()
            try:
                proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                proc.kill()
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            with open(path) as f:
                for line in f:
                    q = [x.strip() for x in line.split(",")]
                    if len(q) < 6:
                        continue
                    try:
                        self.samples.append(float(q[0]))
                        self.max_mhz = float(q[1])
                    except ValueError:
                        continue
                    for nm, v in zip(names, q[2:6]):
                        if v.lower() == "active":
                            self.reasons.add(nm)
            os.unlink(path)
        if not self.samples:
            return None
        return {"sm_mhz": statistics.median(self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(self.samples)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


# the batched frame: the full IW frame, and a small one (1 subswath x 3 bursts
# at half size, default tuning) for quick runs and profiler captures
FRAME_CONFIGS = ("frame", "frame_small")
FRAME_SEED = 20261203 + 2000


def frame_scene(config, rank, device, boxes_of, slc_pairs=None, ground_locked=False):
    """The frame workload of both arms: the seeded synthetic frame on a DEM
    grid where the reference geo2rdr runs of burst pair 0 stay inside their
    buffers (both arms time the same frame on the same grid).
    ``boxes_of(acq)``: the bursts' footprint boxes (the library's planner in
    the s1b arm, the oracle's restatement in the reference arm; the grid
    search gives the same grid for either).  ``slc_pairs``: make the SLCs of
    the first pairs only.  ``ground_locked``: each pair's dates see one scene
    (``synth.ground_lock_pairs``, made on that grid's DEM; needs CUDA and the
    s1b library), else radar-coordinate speckle."""
    from sentinel_gpu_processor_b200 import synth
    small = config == "frame_small"
    sc = synth.make_frame(seed=FRAME_SEED + rank, device=device, slc_pairs=0 if ground_locked else slc_pairs,
                          **(dict(n_swaths=1, n_bursts=3, scale=0.5) if small else {}))
    sc = synth.on_reference_safe_grid(sc, boxes_of, pairs=(0,))
    if ground_locked:
        synth.ground_lock_pairs(sc, range(len(sc.ref) if slc_pairs is None else slc_pairs))
    return sc


def write_pair0(args):
    """``--write-pair0 DIR``: burst pair 0's ground-locked SLCs as the s1b arm
    makes them, written for the reference arm, whose own process must not
    map the s1b library."""
    import numpy as np
    import torch

    from sentinel_gpu_processor_b200 import plan as _plan
    sc = frame_scene(args.config, 0, torch.device("cuda", 0), _plan.footprint_boxes, slc_pairs=1, ground_locked=True)
    np.save(os.path.join(args.write_pair0, "ref.npy"), sc.ref_slc[0].cpu().numpy())
    np.save(os.path.join(args.write_pair0, "sec.npy"), sc.sec_slc[0].cpu().numpy())


def frame_config(args, sc, world):
    """``config`` of the frame workload: the same dict in both arms."""
    small = args.config == "frame_small"
    n = len(sc.ref)
    head = (f"small frame: {n} burst pairs (1 subswath x 3) of half-size bursts" if small else
            f"full IW frame: {n} burst pairs (3 subswaths x 9) of uneven size, lines 1480-1530, samples "
            f"20000-25500, 100-line overlap, Doppler rate per subswath in -1700..-1400 Hz/s, coherence per "
            f"burst in 0.3..0.9")
    samples = "complex int16" if args.samples == "ci16" else "complex64"
    r = sc.rsc
    return {"workload": f"{head}; {samples} SLC samples (band-limited speckle, each pair's dates seeing one scene "
                        f"at their own sample positions); int16 fBm DEM (0-3000 m) on a 1/7200-degree grid",
            "seed": int(sc.seed), "burst_pairs": n,
            "burst_px_per_step": int(sum(a.radar.lines_per_burst * a.radar.samples_per_burst for a in sc.ref)),
            "slc_samples": samples, "looks": [sc.rowlook, sc.collook],
            "goldstein": {"alpha": sc.alpha, "n_win": 32, "step": 8},
            "dem_grid": {"nlat": r.nlat, "nlon": r.nlon, "latmax": r.latmax, "lonmin": r.lonmin, "dlat": r.dlat,
                         "dlon": r.dlon},
            "l2": "inputs larger than L2 (>= 160 MB per burst, read once per step)",
            "parallelism": f"replicas{world}"}


def make_scene(config, seed, device):
    from sentinel_gpu_processor_b200 import synth
    return synth.make_pair(config, seed=seed, device=device)


# ----------------------------------------------------------------------------
# CPU baseline: the float64 oracle on a bounded sample of the same workload
# ----------------------------------------------------------------------------

# the CPU baseline's unit of work: one burst pair of the frame's geometry and
# processing (looks 4 x 20, Goldstein alpha 0.5), 256 lines x 1024 samples
CPU_PAIR = dict(lines=256, samples=1024, rowlook=4, collook=20, alpha=0.5)


def _cpu_pair_worker(seed):
    """The float64 oracle chain on one seeded burst pair, in a spawned worker
    process with one thread: geo2rdr of both SLCs, crossmul + looks, amplitude
    looks and coherence, Goldstein.  Returns (burst pixels, seconds)."""
    for v in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[v] = "1"
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import numpy as np
    import torch
    torch.set_num_threads(1)

    from oracle import coherence as oc
    from oracle import crossmul as ox
    from oracle import geo2rdr as og2
    from oracle import goldstein as ogs
    from sentinel_gpu_processor_b200 import synth
    if seed is None:  # warm-up: imports only
        return 0, 0.0
    sc = synth.make_pair("c0", seed=seed, **CPU_PAIR)
    rsc = og2.Rsc(**sc.rsc.__dict__)
    t0 = time.perf_counter()
    outs = []
    for acq, slc in ((sc.ref[0], sc.ref_slc[0]), (sc.sec[0], sc.sec_slc[0])):
        r = og2.Radar(**{k: getattr(acq.radar, k) for k in og2.Radar.__dataclass_fields__})
        b = og2.BurstMeta(**{k: getattr(acq.bursts[0], k) for k in og2.BurstMeta.__dataclass_fields__})
        outs.append(og2.geo2rdr_burst(slc.numpy(), sc.dem.numpy(), rsc, r, acq.orbit, acq.fm, acq.dc, b))
    (h1, d1), (h2, d2) = outs
    box = ox.intersection_box(h1, h2, sc.rowlook, sc.collook)
    ifg = ox.crossmul_looks(ox.crop(h1, d1, box), ox.crop(h2, d2, box), sc.rowlook, sc.collook)
    a1 = np.sqrt(oc.powlooks(ox.crop(h1, d1, box), sc.rowlook, sc.collook))
    a2 = np.sqrt(oc.powlooks(ox.crop(h2, d2, box), sc.rowlook, sc.collook))
    oc.coherence(ifg, a1, a2)
    if min(ifg.shape) >= 32:
        ogs.goldstein(ifg, 32, sc.alpha)
    return sc.burst_pixels, time.perf_counter() - t0


def cpu_baseline():
    """The float64 NumPy oracle chain on the host's cores: one spawned worker
    per core (spawned, so no worker inherits this process's CUDA context),
    each running the whole chain on its own seeded burst pair; the rate is
    the pixels of all pairs over the wall time of the batch."""
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    ctx = mp.get_context("spawn")
    with ctx.Pool(cores) as pool:
        pool.map(_cpu_pair_worker, [None] * cores)  # workers started and modules imported before timing
        seeds = [20261203 + 4000 + k for k in range(cores)]
        t0 = time.perf_counter()
        res = pool.map(_cpu_pair_worker, seeds, chunksize=1)
        wall = time.perf_counter() - t0
    px = sum(r[0] for r in res)
    busy = sum(r[1] for r in res)
    return {"value": px / wall, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"float64 NumPy oracle chain (geo2rdr x2, crossmul + looks, amplitude looks + coherence, "
                       f"Goldstein) on {cores} seeded burst pairs of {CPU_PAIR['lines']} x {CPU_PAIR['samples']} "
                       f"of the frame's geometry and processing, one per worker process, {cores} processes; "
                       f"{px} burst px in {wall:.1f} s wall ({busy / max(len(res), 1):.1f} s per pair)"),
            "os_cpu_count": os.cpu_count()}


# ----------------------------------------------------------------------------
# s1b arm
# ----------------------------------------------------------------------------

def _workload(args, rank, dev):
    """(scene, chain, run(), host-buffer run maker, description) for the config."""
    from sentinel_gpu_processor_b200 import synth
    from sentinel_gpu_processor_b200.chain import FrameChain, PairChain
    if args.config in FRAME_CONFIGS:
        import torch

        from sentinel_gpu_processor_b200.chain import BatchedFrameChain
        from sentinel_gpu_processor_b200 import plan as _plan
        small = args.config == "frame_small"
        sc = frame_scene(args.config, rank, dev, _plan.footprint_boxes, ground_locked=True)
        chain = BatchedFrameChain(sc.ref, sc.sec, sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=dev,
                                  sample_format=args.samples, deramp_fused=args.deramp == "fused",
                                  crossmul_fused=args.crossmul == "fused")
        if args.samples == "ci16":
            for v, s in zip(chain.ref_views + chain.sec_views, sc.ref_slc + sc.sec_slc):
                v.copy_(synth.cint16(s))
        else:
            chain.load(sc.ref_slc, sc.sec_slc)
        torch.cuda.synchronize()
        sc.ref_slc = sc.sec_slc = None  # the frame's SLC buffer holds them now
        chain.tuned = chain.tuning() if small else chain.autotune(sc.dem, reps=2)
        chain.capture(sc.dem)
        if small:
            head = (f"small frame: {chain.n_pairs} burst pairs (1 subswath x 3) of half-size bursts, default "
                    f"tile shapes")
        else:
            head = (f"full IW frame: {chain.n_pairs} burst pairs (3 subswaths x 9) of uneven size, lines 1480-1530, "
                    f"samples 20000-25500, 100-line overlap; tile shapes from the autotuner")
        desc = (head + f"; batched: one launch per stage over the descriptor table of all {2 * chain.n_pairs} "
                f"bursts, one CUDA graph per step; "
                + ("SLC samples complex int16 (the measurement TIFF's type, widened on the GPU)"
                   if args.samples == "ci16" else "SLC samples complex64 (as the reference's geo2rdr pipe)"))
        return sc, chain, chain.replay, desc
    if args.config == "frame_pairs":
        sc = synth.make_frame(seed=20261203 + 2000 + rank, device=dev)
        chain = FrameChain(sc.ref, sc.sec, sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=dev)
        ins = (sc.ref_slc, sc.sec_slc, sc.dem)
        desc = (f"full IW frame: {len(sc.ref)} burst pairs (3 subswaths x 9) of uneven size, lines 1480-1530, "
                f"samples 20000-25500, 100-line overlap; pair by pair (one host synchronisation per pair)")
        return sc, chain, lambda: chain.run(*ins), desc
    if args.config == "c1":
        from sentinel_gpu_processor_b200.chain import RadarChain
        sc = synth.make_radar_pair("c1", seed=20261203 + 1000 + rank, device=dev)
        chain = RadarChain(sc.ref, sc.sec, sc.ref_slc.shape[0], sc.ref_slc.shape[1], sc.rowlook, sc.collook,
                           sc.alpha, device=dev)
        ins = (sc.ref_slc, sc.sec_slc, sc.lat, sc.lon, sc.hgt)
        chain.capture(*ins)
        desc = (f"one IW burst pair {sc.ref_slc.shape[0]} x {sc.ref_slc.shape[1]} complex64 with float64 lat/lon/hgt "
                "rasters of the reference grid; 8-tap sinc resampling, 5 x 5 coherence; one CUDA graph per step")
        return sc, chain, chain.replay, desc
    sc = make_scene("c1" if args.config == "c1geo" else args.config, 20261203 + 1000 + rank, dev)
    chain = PairChain(sc.ref[0], sc.sec[0], sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=dev)
    ins = (sc.ref_slc[0], sc.sec_slc[0], sc.dem)
    p0 = chain.plans[0]
    desc = (f"one IW burst pair {p0.lines} x {p0.samples} complex64, geocoded on the DEM grid as the reference "
            f"does") if args.config == "c1geo" else f"burst pair {p0.lines} x {p0.samples} ({args.config})"
    return sc, chain, lambda: chain.run(*ins), desc


def _e2e(chain, sc, args, world):
    """End-to-end rate through host buffers: pinned H2D of every SLC and the DEM,
    the chain, D2H of ifg/amplitudes/coherence/filtered ifg, per step."""
    import torch
    if args.config == "c1":
        return _e2e_radar(chain, sc, args, world)
    if args.config in FRAME_CONFIGS:
        return _e2e_frame(chain, sc, args, world)
    frame = args.config == "frame_pairs"
    refs = sc.ref_slc if frame else sc.ref_slc[:1]
    secs = sc.sec_slc if frame else sc.sec_slc[:1]
    ref_h = [t.cpu().pin_memory() for t in refs]
    sec_h = [t.cpu().pin_memory() for t in secs]
    dem_h = sc.dem.cpu().pin_memory()
    ref_d = [torch.empty_like(t, device=chain.dev) for t in ref_h]
    sec_d = [torch.empty_like(t, device=chain.dev) for t in sec_h]
    dem_d = torch.empty_like(dem_h, device=chain.dev)
    host_out = {}
    h2d = sum(t.numel() * t.element_size() for t in ref_h + sec_h) + dem_h.numel() * dem_h.element_size()

    def step():
        dem_d.copy_(dem_h, non_blocking=True)
        d2h = 0
        for k in range(len(ref_h)):
            ref_d[k].copy_(ref_h[k], non_blocking=True)
            sec_d[k].copy_(sec_h[k], non_blocking=True)
            res = chain.run_pair(k, ref_d[k], sec_d[k], dem_d) if frame else chain.run(ref_d[k], sec_d[k], dem_d)
            if res is None:
                continue
            for name in ("ifg", "amp1", "amp2", "coh", "filt"):
                v = getattr(res, name)
                key = (k, name)
                if key not in host_out or host_out[key].shape != v.shape:
                    host_out[key] = torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                host_out[key].copy_(v, non_blocking=True)
                d2h += v.numel() * v.element_size()
        torch.cuda.current_stream().synchronize()
        return d2h

    step()
    k_e2e = max(3, args.steps // 4) if frame else max(3, args.steps // 2)
    barrier(world)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    d2h = 0
    for _ in range(k_e2e):
        d2h = step()
    t2.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(s2.elapsed_time(t2), world)
    return job_rate(world, k_e2e, chain.burst_pixels, e2e_ms), h2d, d2h


def _e2e_frame(chain, sc, args, world):
    """End to end for the batched frame through ``FramePipeline``: per frame
    the pinned H2D of every burst of both acquisitions and of the DEM, the
    frame run (graph replay) and the D2H of the product arrays (ifg,
    amplitudes, coherence, filtered ifg).  Frames alternate between two input
    slots, so the H2D of frame k + 1 (copy stream) overlaps frame k's run;
    every frame's copies are inside the timed region."""
    import torch

    from sentinel_gpu_processor_b200.chain import FramePipeline
    host_in = [v.cpu().pin_memory() for v in chain.ref_views + chain.sec_views]
    dem_h = sc.dem.cpu().pin_memory()
    pipe = FramePipeline(chain, sc.dem)
    host_out = [torch.empty(o.shape, dtype=o.dtype, pin_memory=True) for o in pipe.outputs()]
    h2d = sum(t.numel() * t.element_size() for t in host_in) + dem_h.numel() * dem_h.element_size()
    d2h = sum(t.numel() * t.element_size() for t in host_out)

    def step():
        pipe.submit(host_in, dem_h, host_out)

    step()
    step()  # both slots warm
    torch.cuda.synchronize()
    k_e2e = max(3, args.steps // 4)
    barrier(world)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    pipe.copy.wait_event(s2)  # no copy starts before the timed region
    for _ in range(k_e2e):
        step()
    t2.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(s2.elapsed_time(t2), world)
    return job_rate(world, k_e2e, chain.burst_pixels, e2e_ms), h2d, d2h


def _e2e_radar(chain, sc, args, world):
    """End to end for the radar-grid chain: pinned H2D of both SLCs and the
    float64 lat/lon/height rasters into the graph's input tensors, graph
    replay, D2H of ifg, amplitudes, looked and full-resolution coherence and
    the filtered ifg."""
    import torch
    dev_ins = (sc.ref_slc, sc.sec_slc, sc.lat, sc.lon, sc.hgt)
    host_ins = [t.cpu().pin_memory() for t in dev_ins]
    h2d = sum(t.numel() * t.element_size() for t in host_ins)
    outs = chain.outs
    names = ("ifg", "amp1", "amp2", "coh", "filt", "coh_full")
    host_out = {n: torch.empty(outs[n].shape, dtype=outs[n].dtype, pin_memory=True) for n in names}
    d2h = sum(t.numel() * t.element_size() for t in host_out.values())

    def step():
        for d, h in zip(dev_ins, host_ins):
            d.copy_(h, non_blocking=True)
        chain.replay()
        for n in names:
            host_out[n].copy_(outs[n], non_blocking=True)
        torch.cuda.current_stream().synchronize()

    step()
    k_e2e = max(3, args.steps // 2)
    barrier(world)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(k_e2e):
        step()
    t2.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(s2.elapsed_time(t2), world)
    return job_rate(world, k_e2e, chain.burst_pixels, e2e_ms), h2d, d2h


KERNELS = ("deramp", "geo2rdr", "crossmul_looks", "goldstein", "geo2rdr_offsets", "resample", "box_coherence")


def _instrumented(run, steps):
    """Per-entry-point device times over ``steps`` eager steps: the library call
    of every s1b entry point is bracketed by CUDA events on the current stream
    (kernels.timer hook).  Returns {name: [ms, ...]}."""
    import contextlib

    import torch

    from sentinel_gpu_processor_b200 import kernels as K
    rec = {}

    @contextlib.contextmanager
    def timer(name):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        yield
        e1.record()
        rec.setdefault(name, []).append((e0, e1))

    K.timer = timer
    try:
        for _ in range(steps):
            run()
        torch.cuda.synchronize()
    finally:
        K.timer = None
    return {n: [a.elapsed_time(b) for a, b in v] for n, v in rec.items() if n in KERNELS}


def _radar_inputs(sc):
    return (sc.ref_slc, sc.sec_slc, sc.lat, sc.lon, sc.hgt)


def _kernel_table(chain, sc, args, times, peak):
    """Algorithmic bytes per launch and achieved GB/s for each entry point."""
    rows = {}
    if args.config == "c1":
        px = chain.burst_pixels
        ml = (chain.box[3] // chain.rowlook) * (chain.box[2] // chain.collook)
        box_px = chain.box[2] * chain.box[3]
        bytes_per = {"geo2rdr_offsets": 32 * px, "resample": 24 * px, "crossmul_looks": 16 * box_px + 20 * ml,
                     "box_coherence": 20 * px, "goldstein": 16 * ml}
    elif args.config in FRAME_CONFIGS:
        # one launch per stage covers every burst / pair of the frame
        pls = chain.plans
        burst = sum(p.lines * p.samples for p in pls)
        geo = sum(p.nrow * p.ncol for p in pls)
        res = [r for r in chain.last if r is not None]
        box_px = sum((r.box[2] - r.box[0]) * (r.box[3] - r.box[1]) for r in res)
        ml = sum(r.ifg.numel() for r in res)
        # deramp: read one input sample (8 bytes complex64, 4 complex int16), write 8;
        # fused, the stage only writes the column tables (16 bytes per column) and
        # the geocoding reads the raw samples instead of the deramped copy
        din = 4 if getattr(chain, "sample_format", "c64") == "ci16" else 8
        if getattr(chain, "deramp_fused", False):
            cols = sum(p.samples for p in pls)
            if "deramp" in times:
                times["tops_table"] = times.pop("deramp")
            bytes_per = {"tops_table": 16 * cols, "geo2rdr": GEO_BYTES_PER_GEO_PX * geo + din * burst + 16 * cols}
        else:
            bytes_per = {"deramp": (din + 8) * burst,
                         "geo2rdr": GEO_BYTES_PER_GEO_PX * geo + GEO_BYTES_PER_BURST_PX * burst}
        bytes_per.update({"crossmul_looks": 16 * box_px + 20 * ml, "goldstein": 16 * ml})
        if getattr(chain, "crossmul_fused", False):
            # the geocoding reads each DEM height once per pair and writes one
            # float4 of look sums per column and look row of the pair's union
            # window instead of both geocoded windows; the crossmul stage reads
            # the sums over the box
            rl = chain.rowlook
            union = 0
            for a, b in zip(pls[0::2], pls[1::2]):
                top = min(a.win_top, b.win_top) // rl * rl
                n_rows = -(-(max(a.win_bottom, b.win_bottom) - top) // rl) * rl
                union += n_rows * (max(a.win_right, b.win_right) - min(a.win_left, b.win_left))
            geo_in = bytes_per["geo2rdr"] - GEO_BYTES_PER_GEO_PX * geo
            bytes_per["geo2rdr"] = geo_in + 2 * union + 16 * union // rl
            bytes_per["crossmul_looks"] = 16 * box_px // rl + 20 * ml
    else:
        pls = [p for pl in chain.pairs for p in pl] if args.config == "frame_pairs" else chain.plans
        n = len(pls)
        burst = sum(p.lines * p.samples for p in pls) / n
        geo = sum(p.nrow * p.ncol for p in pls) / n
        bytes_per = {"deramp": 16 * burst, "geo2rdr": GEO_BYTES_PER_GEO_PX * geo + GEO_BYTES_PER_BURST_PX * burst}
        if args.config == "frame_pairs":
            res = [r for r in chain.last if r is not None]
            box_px = sum((r.box[2] - r.box[0]) * (r.box[3] - r.box[1]) for r in res) / len(res)
            ml = sum(r.ifg.numel() for r in res) / len(res)
        else:
            r = chain.last
            box_px = (r.box[2] - r.box[0]) * (r.box[3] - r.box[1])
            ml = r.ifg.numel()
        bytes_per.update({"crossmul_looks": 16 * box_px + 20 * ml, "goldstein": 16 * ml})
    for name, ts in times.items():
        if name not in bytes_per:
            continue
        ms = sum(ts) / len(ts)
        gbs = bytes_per[name] / (ms / 1e3) / 1e9
        rows[name] = {"launches": len(ts), "avg_ms": ms, "total_ms": sum(ts), "bytes_per_launch": bytes_per[name],
                      "achieved_gbs": gbs, "frac": gbs / peak}
    return rows


def _timed_replays(run, steps, warm=3):
    """ms per step of ``run`` over ``steps`` steps, CUDA events on the current stream."""
    import torch
    for _ in range(warm):
        run()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        run()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps


def _ci16_variant(chain, sc, steps):
    """The same frame from complex int16 samples (the measurement TIFF's type,
    round(2000 s), widened on the GPU), with the complex64 run's tile shapes:
    device-resident rate."""
    import torch

    from sentinel_gpu_processor_b200 import synth
    from sentinel_gpu_processor_b200.chain import BatchedFrameChain
    v = BatchedFrameChain(sc.ref, sc.sec, sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=chain.dev,
                          sample_format="ci16", deramp_fused=chain.deramp_fused, crossmul_fused=chain.crossmul_fused)
    for dst, src in zip(v.ref_views + v.sec_views, chain.ref_views + chain.sec_views):
        dst.copy_(synth.cint16(src))
    v.set_tuning(**chain.tuning())
    v.capture(sc.dem)
    ms = _timed_replays(v.replay, steps)
    del v
    torch.cuda.empty_cache()
    return {"value": chain.burst_pixels / (ms / 1e3), "unit": UNIT, "ms_per_step": ms,
            "slc_samples": "complex int16 (round(2000 s), widened on the GPU)", "tuning": chain.tuning()}


def _radar_extras(dev, peak, steps=10):
    """Radar-grid kernels on one 1500 x 21000 burst pair (8-tap sinc
    resampling, 5 x 5 box coherence): per-kernel times from CUDA events
    around each entry point over eager steps, and their HBM fractions."""
    import torch

    from sentinel_gpu_processor_b200 import synth
    from sentinel_gpu_processor_b200.chain import RadarChain
    sc = synth.make_radar_pair("c1", seed=20261203 + 1000, device=dev)
    chain = RadarChain(sc.ref, sc.sec, sc.ref_slc.shape[0], sc.ref_slc.shape[1], sc.rowlook, sc.collook, sc.alpha,
                       device=dev)
    ins = _radar_inputs(sc)
    for _ in range(3):
        chain.run(*ins)
    torch.cuda.synchronize()
    if not chain.staging_ok():
        raise SystemExit("a shared-memory staging copy did not complete")
    times = _instrumented(lambda: chain.run(*ins), steps)
    px = chain.burst_pixels
    bytes_per = {"geo2rdr_offsets": 32 * px, "resample": 24 * px, "box_coherence": 20 * px}
    out = {"workload": f"one burst pair {chain.L} x {chain.S} complex64, float64 lat/lon/hgt rasters",
           "peak_gbs": peak}
    for name, b in bytes_per.items():
        ts = times.get(name)
        if not ts:
            continue
        ms = sum(ts) / len(ts)
        gbs = b / (ms / 1e3) / 1e9
        out[name] = {"avg_ms": ms, "bytes_per_launch": b, "achieved_gbs": gbs, "frac": gbs / peak,
                     "launches": len(ts)}
    del chain, sc
    torch.cuda.empty_cache()
    return out


def _workdir(need_bytes):
    """A scratch directory on /dev/shm when it has room, else on disk."""
    base = None
    if os.path.isdir("/dev/shm"):
        st = os.statvfs("/dev/shm")
        if st.f_bavail * st.f_frsize > 2 * need_bytes:
            base = "/dev/shm"
    return tempfile.mkdtemp(prefix="s1b_check_", dir=base)


def parity_leg(pair, dem_host, rsc, looks, alpha, plans, dem_dev):
    """Checker (outside every timed region): burst pair 0 of the frame run
    through the reference executables (sm_100a builds of its sources in
    oracle/_ref: geo2rdr x 2, crossmul_daemon, goldstein) on the same inputs
    in its file formats, and the reference's NumPy amplitude-look and
    coherence formulas on their outputs; compared with the batched frame's
    products of pair 0.  The geocoding's sample coordinates
    (s1b_geo2rdr_grid_offsets) are compared with the float64 oracle on rows
    spread over both bursts' DEM windows.

    ``pair``: dict with the acquisitions, complex64 SLCs (numpy) and the
    frame's products of pair 0 (numpy)."""
    import numpy as np

    from oracle import coherence as oc
    from oracle import crossmul as ox
    from oracle import geo2rdr as og2
    from oracle import refrun
    from sentinel_gpu_processor_b200 import formats, kernels
    out = {"pair": 0}
    rl, cl = looks
    # sample coordinates of the geocoding against the float64 oracle
    off = {}
    for tag, acq, pl in (("ref", pair["ref"], plans[0]), ("sec", pair["sec"], plans[1])):
        az, rg = kernels.geo2rdr_grid_offsets(pl, dem_dev)
        rows = np.linspace(0, pl.nrow - 1, 8).round().astype(np.int64)
        r = og2.Radar(**{k: getattr(acq.radar, k) for k in og2.Radar.__dataclass_fields__})
        b = og2.BurstMeta(**{k: getattr(acq.bursts[0], k) for k in og2.BurstMeta.__dataclass_fields__})
        win = dem_host[pl.win_top:pl.win_bottom, pl.win_left:pl.win_right]
        oaz, org = og2.window_offsets(win, rows, r, acq.orbit, b, rsc.latmax + rsc.dlat * pl.win_top,
                                      rsc.lonmin + rsc.dlon * pl.win_left, rsc.dlat, rsc.dlon)
        gaz, grg = az.cpu().numpy()[rows], rg.cpu().numpy()[rows]
        used = ((org > b.first_valid_sample) & (org < b.last_valid_sample - 1) & (oaz >= b.first_valid_line + 5)
                & (oaz < b.last_valid_line - 5))
        off[tag] = {"rows": int(len(rows)), "pixels": int(oaz.size), "pixels_in_burst": int(used.sum()),
                    "max_az_px": float(np.abs(gaz - oaz)[used].max()) if used.any() else None,
                    "max_rg_px": float(np.abs(grg - org)[used].max()) if used.any() else None,
                    "max_az_px_whole_window": float(np.abs(gaz - oaz).max()),
                    "max_rg_px_whole_window": float(np.abs(grg - org).max())}
        del az, rg
    vals = [v for t in off.values() for v in (t["max_az_px"], t["max_rg_px"]) if v is not None]
    out["offset_px"] = max(vals) if vals else None
    out["offsets_vs_float64_oracle"] = off
    if not refrun.available():
        out["reference"] = "unavailable: reference executables not built in oracle/_ref"
        return out
    wd = _workdir(dem_host.nbytes + 2 * pair["ref_slc"].nbytes)
    try:
        rscf, demf = refrun.write_dem(wd, rsc, dem_host)
        gs = {}
        for tag in ("ref", "sec"):
            db = refrun.write_geo2rdr_inputs(wd, tag, pair[tag], [pair[tag + "_slc"]], rscf, demf)
            o, _ = refrun.geo2rdr(db, os.path.join(wd, tag), 1)
            gs[tag] = o[0]
        f1, f2 = os.path.join(wd, "ref_burst_0.gslc"), os.path.join(wd, "sec_burst_0.gslc")
        fo = os.path.join(wd, "pair.int")
        refrun.crossmul_daemon([(f1, f2, fo)], os.path.join(wd, "tasks.txt"), rl, cl, manual=False)
        wh, wifg = formats.read_raster(fo)
        (h1, d1), (h2, d2) = gs["ref"], gs["sec"]
        box = (int(wh[2]) * cl, int(wh[3]) * rl, int(wh[4]) * cl, int(wh[5]) * rl)
        wa1 = np.sqrt(oc.powlooks(ox.crop(h1, d1, box), rl, cl))
        wa2 = np.sqrt(oc.powlooks(ox.crop(h2, d2, box), rl, cl))
        with np.errstate(divide="ignore", invalid="ignore"):
            wc = np.abs(wifg) / (wa1 + 1e-12) / (wa2 + 1e-12)
        gf = os.path.join(wd, "ifg.int")
        np.ascontiguousarray(wifg, dtype=np.complex64).tofile(gf)
        wfilt, _ = refrun.goldstein(gf, wifg.shape[0], wifg.shape[1], 32, alpha)
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    ifg, a1, a2, coh, filt = (pair[k] for k in ("ifg", "amp1", "amp2", "coh", "filt"))
    gh = np.asarray(pair["header"][:6])
    out["ifg_header_equal"] = bool(np.array_equal(gh, np.asarray(wh[:6])))
    out["ifg_headers"] = {"ours": [int(v) for v in gh], "reference": [int(v) for v in wh[:6]]}
    out["gslc_crop_rows"] = {"ours": [[int(h[3]), int(h[5])] for h in pair["gslc_headers"]],
                             "reference": [[int(h1[3]), int(h1[5])], [int(h2[3]), int(h2[5])]]}
    # common multilooked region of the two interferograms (the reference's crop
    # rows can be narrower, geo2rdr.cu:115-122; every row of its box is one it
    # kept, so the common region holds identical inputs)
    l0, t0 = max(gh[2], wh[2]), max(gh[3], wh[3])
    r0, b0 = min(gh[4], wh[4]), min(gh[5], wh[5])
    if r0 <= l0 or b0 <= t0:
        out["common_region"] = "empty"
        return out

    def cut(a, h):
        return a[t0 - h[3]:b0 - h[3], l0 - h[2]:r0 - h[2]]

    ifg_c, a1_c, a2_c, coh_c = (cut(x, gh) for x in (ifg, a1, a2, coh))
    wifg_c, wa1_c, wa2_c, wc_c = (cut(x, wh) for x in (wifg, wa1, wa2, wc))
    out["common_ml_pixels"] = int(ifg_c.size)
    both = (np.abs(ifg_c) > 0) & (np.abs(wifg_c) > 0)
    d = np.angle(ifg_c[both].astype(np.complex128) * np.conj(wifg_c[both].astype(np.complex128)))
    out["rms_phase_rad"] = float(np.sqrt(np.mean(d * d))) if d.size else None
    out["ifg_rel_err"] = float(np.abs(ifg_c.astype(np.complex128) - wifg_c).max() / np.abs(wifg_c).max())
    out["validity_mismatch_frac"] = float(((np.abs(ifg_c) > 0) != (np.abs(wifg_c) > 0)).mean())
    out["amp_rel_err"] = float(max(np.abs(a1_c - wa1_c).max() / wa1_c.max(), np.abs(a2_c - wa2_c).max() / wa2_c.max()))
    # coherence: pixels where neither side takes the > 1 fill (seeded here,
    # unseeded rand() in the reference)
    with np.errstate(divide="ignore", invalid="ignore"):
        raw = np.abs(ifg_c.astype(np.complex128)) / (a1_c + 1e-12) / (a2_c + 1e-12)
    m = both & np.isfinite(wc_c) & (wc_c <= 1.0) & (raw <= 1.0)
    out["max_dcoh"] = float(np.abs(coh_c[m] - wc_c[m]).max()) if m.any() else None
    if out["ifg_header_equal"]:
        gfilt, src = filt, "the frame's own interferogram"
    else:  # the patch grids differ with the image extent: filter the reference's interferogram
        import torch

        from sentinel_gpu_processor_b200 import kernels as K
        gfilt = K.goldstein(torch.from_numpy(np.ascontiguousarray(wifg, dtype=np.complex64)).cuda(), alpha).cpu().numpy()
        src = "the reference's interferogram (headers differ)"
    fm = (np.abs(gfilt) > 0) & (np.abs(wfilt) > 1e-3 * np.abs(wfilt).max())
    d = np.angle(gfilt[fm].astype(np.complex128) * np.conj(wfilt[fm].astype(np.complex128)))
    out["goldstein_rms_phase_rad"] = float(np.sqrt(np.mean(d * d))) if d.size else None
    out["goldstein_input"] = src
    out["against"] = ("reference executables geo2rdr x2, crossmul_daemon, goldstein (cuFFT), sm_100a builds of its "
                      "sources, and its NumPy amplitude-look and coherence formulas; same inputs in its file formats")
    out["tolerances"] = {"rms_phase_rad": 1e-3, "max_dcoh": 1e-4, "offset_px": 1e-4}
    return out


def run_s1b(args):
    import torch
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    sc, chain, run, desc = _workload(args, rank, dev)
    frame = args.config in FRAME_CONFIGS
    warm = max(args.warmup, 3)
    res = None
    for _ in range(warm):
        res = run()
    torch.cuda.synchronize()
    if frame:
        res = chain.results()
    if res is None or (isinstance(res, list) and any(r is None for r in res)):
        raise SystemExit("empty interferogram for the synthetic input")
    if hasattr(chain, "staging_ok") and not chain.staging_ok():
        raise SystemExit("a shared-memory staging copy did not complete")
    stream = torch.cuda.current_stream()
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        out = run()
        res = res if out is None else out
    stop.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    chain.geo_events = None
    barrier(world)
    elapsed_ms = max_over_ranks(start.elapsed_time(stop), world)
    value = job_rate(world, args.steps, chain.burst_pixels, elapsed_ms)
    e2e, h2d, d2h = _e2e(chain, sc, args, world)
    chain.last = res
    peak, peak_kind = peaks()
    if frame:
        times = {}
        for _ in range(max(2, min(args.steps, 10))):
            for name, ms in chain.profile(sc.dem).items():
                times.setdefault(name, []).append(ms)
    else:
        times = _instrumented(run if args.config != "c1" else (lambda: chain.run(*_radar_inputs(sc))),
                              max(2, min(args.steps, 10)))
    table = _kernel_table(chain, sc, args, times, peak)
    top = max(table, key=lambda n: table[n]["total_ms"])
    run_info = {"implementation": desc}
    if frame:
        run_info.update({"geo_px_total": sum(chain.geo_pixels()),
                         "ifg_ml_shapes_first3": [list(r.ifg.shape) for r in res[:3]],
                         # simulated and measured (valid cells) coherence of every pair
                         "coherence_sim_per_pair": [round(g, 3) for g in sc.extra["coherence"]],
                         "mean_coherence_per_pair": [None if r is None else round(_mean_valid(r.coh), 3)
                                                     for r in res],
                         "batched": True, "cuda_graph": True, "tuning": chain.tuned,
                         "tuning_source": chain.tuning_source,
                         "deramp": "fused into the geocoding gathers" if chain.deramp_fused else "separate kernel",
                         "crossmul": ("look sums formed in the geocoding (no geocoded windows)"
                                      if chain.crossmul_fused else "kernel reading the geocoded windows")})
        launches = chain.launches_per_step()
    elif args.config == "frame_pairs":
        run_info.update({"burst_pairs": len(chain.pairs), "burst_px_per_step": chain.burst_pixels,
                         "geo_px_total": sum(chain.geo_pixels()),
                         "ifg_ml_shapes_first3": [list(r.ifg.shape) for r in res[:3]], "batched": False})
        launches = chain.launches_per_step()
    elif args.config == "c1":
        run_info.update({"lines": chain.L, "samples": chain.S, "ifg_ml": list(res["ifg"].shape),
                         "interp": chain.interp, "coherence_window": chain.win, "cuda_graph": True})
        launches = chain.launches_per_step()
    else:
        run_info.update({"lines": chain.plans[0].lines, "samples": chain.plans[0].samples,
                         "geo_px_total": sum(p.nrow * p.ncol for p in chain.plans), "ifg_ml": list(res.ifg.shape)})
        launches = chain.launches_per_step()
    traffic = None
    if top == "geo2rdr":
        if frame:  # one launch geocodes every burst
            if chain.crossmul_fused:
                ratio = GEO_XMUL_TRAFFIC_RATIO.get(args.samples)
                traffic = ratio * table["geo2rdr"]["bytes_per_launch"] if ratio and chain.deramp_fused else None
            else:
                traffic = (GEO_FUSED_TRAFFIC_RATIO * table["geo2rdr"]["bytes_per_launch"] if chain.deramp_fused
                           else GEO_DRAM_BYTES_PER_GEO_PX * sum(p.nrow * p.ncol for p in chain.plans))
        else:
            pls = [p for pl in chain.pairs for p in pl] if args.config == "frame_pairs" else chain.plans
            traffic = GEO_DRAM_BYTES_PER_GEO_PX * sum(p.nrow * p.ncol for p in pls) / len(pls)
    elif top == "resample":
        traffic = RESAMPLE_DRAM_BYTES_PER_PX * chain.burst_pixels
    if frame:
        cfg = frame_config(args, sc, world)
    else:
        cfg = {"workload": desc, "looks": [sc.rowlook, sc.collook],
               "goldstein": {"alpha": sc.alpha, "n_win": 32, "step": 8},
               "l2": "inputs larger than L2 (>= 252 MB per SLC, read once per step)",
               "parallelism": f"replicas{world}"}
    t = table[top]
    samples = "ci16 input widened to c64" if (frame and args.samples == "ci16") else "c64"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": warm, "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": f"f64 geometry + {samples}", "data": "synthetic",
        "config": cfg, "run": run_info,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches * args.steps,
        "roofline": {"bound": "hbm", "kernel": top, "achieved": t["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": t["frac"], "traffic": traffic, "peak_kind": peak_kind,
                     "bytes_per_launch": t["bytes_per_launch"], "launch_ms": t["avg_ms"],
                     "timed": ("CUDA events between the stages of profiled frame runs" if frame
                               else "CUDA events around every launch of the entry point over instrumented eager steps"),
                     "limiter": GEO_LIMITER if top == "geo2rdr" else "HBM"},
        "kernels": table,
    }
    if frame and top == "geo2rdr" and chain.crossmul_fused and chain.deramp_fused:
        # the geocoding's FP64 work against the GPU's measured FP64 throughput
        flop = GEO_FP64_FLOP_PER_GEO_PX * run_info["geo_px_total"]
        ach = flop / (t["avg_ms"] * 1e-3) / 1e12
        pk = fp64_peak_tflops(dev)
        line["roofline"]["fp64"] = {
            "flop_per_launch": flop, "achieved_tflops": ach, "peak_tflops": pk, "frac": ach / pk,
            "peak_kind": "measured: torch float64 matmul 4096^3, best of 5",
            "count": f"at most {GEO_FP64_FLOP_PER_GEO_PX} FP64 operations per geocoded DEM pixel (ncu per-opcode "
                     f"counts: 2 DFMA + DMUL + DADD, before the last loop hoists) x geocoded pixels"}
    if clk is not None:
        line["clocks"] = clk
    checker = rank == 0 and world == 1
    pair0 = None
    if frame and checker and not args.no_parity:
        # pair 0's inputs and products, kept on the host for the checker leg
        p0 = res[0]
        views = (chain.ref_views[0], chain.sec_views[0])
        if chain.sample_format == "ci16":
            views = tuple(torch.view_as_complex(v.float()) for v in views)
        pair0 = {"ref": sc.ref[0], "sec": sc.sec[0], "ref_slc": views[0].cpu().numpy(),
                 "sec_slc": views[1].cpu().numpy(), "header": list(p0.header[:6]),
                 "gslc_headers": [list(h[:6]) for h in p0.gslc_headers],
                 **{k: getattr(p0, k).cpu().numpy() for k in ("ifg", "amp1", "amp2", "coh", "filt")}}
        plans0 = (chain.plans[0], chain.plans[1])
    if frame and not args.no_extras:
        extras = {"complex_int16": _ci16_variant(chain, sc, args.steps)}
        line["value_ci16"] = extras["complex_int16"]["value"]
    if frame:
        res = out = None
        del chain, run
        torch.cuda.empty_cache()
        if not args.no_extras:
            extras["radar_grid_c1"] = _radar_extras(dev, peak)
            extras["adjoint_c3"] = adjoint_measure(dev, max(3, min(args.steps, 10)), world, compact=True)
            # the float64 checker of every pair's sample coordinates runs at N = 1 only
            stack = stack_measure(dev, 3, world, offsets_rows=0 if (args.no_parity or world > 1) else 1)
            by_date, errs = {}, []
            for p in stack.pop("per_pair"):
                if p["mean_coherence"] is not None:
                    by_date.setdefault(p["date"], []).append(p["mean_coherence"])
                if "offset_err_px" in p:  # per pair (date-major): the larger of both bursts' errors
                    errs.append(float(f"{max(p['offset_err_px']['ref'], p['offset_err_px']['sec']):.3g}"))
            stack["mean_coherence_per_date"] = [round(sum(v) / len(v), 4) for _, v in sorted(by_date.items())]
            if errs:
                stack["offset_err_px_per_pair"] = errs
            extras["stack_c4"] = stack
            line["extras"] = extras
        if pair0 is not None:
            line["parity"] = parity_leg(pair0, sc.dem.cpu().numpy(), sc.rsc, (sc.rowlook, sc.collook), sc.alpha,
                                        plans0, sc.dem)
    if checker and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------------------------
# reference arm
# ----------------------------------------------------------------------------

def _repo_libraries_mapped():
    """Shared objects from this repository mapped into this process."""
    try:
        with open("/proc/self/maps") as f:
            paths = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so") or ".so." in ln}
    except OSError:
        return None
    return sorted(p for p in paths if p.startswith(ROOT) and "baseline/_ref" not in p)


def _kbench_inputs(wd, sc, dem, slcs):
    """Inputs of the reference's kernels for burst pair 0, for the
    kernel-only harness (oracle/_ref/bin/kbench_chain): the host-side values
    the reference geo2rdr computes before its launches (geo2rdr.cu:469-613),
    from the oracle's restatement of them, and the raw arrays.  Returns the
    manifest entries (the crossmul box is added once the reference has run)."""
    import numpy as np

    from oracle import geo2rdr as og2
    from oracle import geometry as og
    m = {}
    r = sc.rsc
    orsc = og2.Rsc(nlat=r.nlat, nlon=r.nlon, latmax=r.latmax, lonmin=r.lonmin, dlat=r.dlat, dlon=r.dlon)
    for tag, acq in (("ref", sc.ref[0]), ("sec", sc.sec[0])):
        rad = og2.Radar(**{k: getattr(acq.radar, k) for k in og2.Radar.__dataclass_fields__})
        b = og2.BurstMeta(**{k: getattr(acq.bursts[0], k) for k in og2.BurstMeta.__dataclass_fields__})
        co = og2.burst_coefficients(rad, acq.orbit, acq.fm, acq.dc, b)
        w = og2.dem_window(og2.burst_latlon_box(rad, acq.orbit, b), orsc)
        tt, xx, vv = (np.ascontiguousarray(a, dtype=np.float64) for a in acq.orbit)
        L, S = rad.lines_per_burst, rad.samples_per_burst
        dtaz = 1.0 / rad.prf
        tstart = b.azimuth_time
        tmid = (tstart + (tstart + (L - 1) * dtaz)) * 0.5
        xmid, vmid = og.intp_orbit(tt, xx, vv, np.float64(tmid))
        p = f"{tag}_"
        arrays = {"slc": np.ascontiguousarray(slcs[tag], dtype=np.complex64), "kt": co.kt, "etaref": co.etaref,
                  "eta": co.eta, "tt": tt, "xx": xx, "vv": vv,
                  "dem": np.ascontiguousarray(dem[w.top:w.bottom, w.left:w.right], dtype=np.int16)}
        for name, a in arrays.items():
            path = os.path.join(wd, f"kb_{p}{name}.bin")
            a.tofile(path)
            m[p + name] = path
        m.update({p + "L": L, p + "S": S, p + "nstat": len(tt), p + "nrow": w.nrow, p + "ncol": w.ncol,
                  p + "win_left": w.left, p + "win_top": w.top, p + "fvl": b.first_valid_line,
                  p + "lvl": b.last_valid_line, p + "fvs": b.first_valid_sample, p + "lvs": b.last_valid_sample,
                  p + "tmid": tmid, p + "latmax0": r.latmax + r.dlat * w.top,
                  p + "lonmin0": r.lonmin + r.dlon * w.left, p + "dlat": r.dlat, p + "dlon": r.dlon,
                  p + "rngstart": rad.slant_range_time * 299792458.0 / 2.0,
                  p + "tstart": tstart, p + "dmrg": 299792458.0 / 2.0 / rad.range_sampling_rate, p + "dtaz": dtaz,
                  p + "etac0": co.etac0, p + "ks": co.ks, p + "wvl": rad.wvl})
        for i in range(4):
            m[p + f"fm{i}"] = co.fm[i]
            m[p + f"dc{i}"] = co.dc[i]
        for i in range(3):
            m[p + f"xmid{i}"] = float(xmid[i])
            m[p + f"vmid{i}"] = float(vmid[i])
    return m


def _kbench_run(wd, m, ifg_header, looks, alpha, burst_px, reps=5):
    """The reference's kernels on device-resident inputs (kernel-only
    harnesses oracle/_ref/bin/kbench_chain and kbench_goldstein, built from
    its sources): per-kernel median times for burst pair 0 and the rate they
    give in burst pixels per second."""
    import numpy as np

    from oracle import refrun
    rl, cl = looks
    h = ifg_header
    m = dict(m, box_left=int(h[2]) * cl, box_top=int(h[3]) * rl, box_right=int(h[4]) * cl,
             box_bottom=int(h[5]) * rl, rowlook=rl, collook=cl)
    man = os.path.join(wd, "kbench_manifest.txt")
    with open(man, "w") as f:
        for k, v in m.items():
            if isinstance(v, str):
                f.write(f"{k} {v}\n")
            elif isinstance(v, (int, np.integer)):
                f.write(f"{k} {int(v)}\n")
            else:
                f.write(f"{k} {float(v)!r}\n")
    ifg = os.path.join(wd, "kbench_ifg.bin")
    _, out = refrun.run([os.path.join(refrun.BIN, "kbench_chain"), man, str(reps), ifg])
    chain = json.loads(out.strip().splitlines()[-1])
    nr, nc = chain["ifg_shape"]
    _, out = refrun.run([os.path.join(refrun.BIN, "kbench_goldstein"), ifg, str(nr), str(nc), "32", repr(float(alpha)),
                         str(reps)])
    gold = json.loads(out.strip().splitlines()[-1])
    pair_ms = (sum(chain["deramp_ms"]) + sum(chain["reproject_ms"]) + sum(chain["nonzero_rows_ms"])
               + chain["crossmul_looks_ms"] + gold["goldstein_ms"])
    return {"value": burst_px / (pair_ms / 1e3), "unit": UNIT, "pair_ms": pair_ms,
            "kernels": {"deramp_burst_ms": chain["deramp_ms"], "reproject_ms": chain["reproject_ms"],
                        "find_nonzero_rows_ms": chain["nonzero_rows_ms"],
                        "conj_mul_col_row_look_ms": chain["crossmul_looks_ms"],
                        "goldstein_filter_cuda_host_ms": gold["goldstein_ms"], "cufft_plan_ms": gold["plan_ms"]},
            "geo_px": chain["geo_px"], "ifg_shape": chain["ifg_shape"], "reps": reps,
            "how": ("the reference's kernels (sm_100a builds of its geo2rdr.cu, sario.cu, goldstein.cu) on "
                    "device-resident inputs of burst pair 0, its launch configurations, CUDA events, median of "
                    f"{reps} after a warm-up; no process start-up, SQLite, file I/O or host copies except the "
                    "filtered image's copy inside goldstein_filter_cuda_host")}


def run_reference(args):
    """The reference's own implementation on the same workload: its CUDA
    executables (sm_100a builds of its sources in oracle/_ref) geo2rdr x 2,
    crossmul_daemon and goldstein, and its NumPy amplitude-look and coherence
    formulas, with the inputs in its file formats.  Frame configurations: a
    bounded sample of the frame, burst pair 0, per step (the reference runs
    geo2rdr once per burst for bursts of uneven size).  The scene is built
    without the s1b library (the oracle's footprint boxes pick the same DEM
    grid), so this process maps none of the repository's shared objects."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import numpy as np

    from oracle import coherence as oc
    from oracle import crossmul as ox
    from oracle import refrun
    from sentinel_gpu_processor_b200 import formats
    if not refrun.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference executables not built in oracle/_ref "
                                                              "(python oracle/build_ref.py)"}))
        return
    frame = args.config in FRAME_CONFIGS
    if frame:
        import torch
        dev = "cuda" if torch.cuda.is_available() else "cpu"
        sc = frame_scene(args.config, 0, dev, refrun.footprint_boxes, slc_pairs=0)
        cfg = frame_config(args, sc, world)
        dem = sc.dem.cpu().numpy()
        # burst pair 0's SLCs come from a process of their own (they are made
        # with s1b kernels, which this process must not map)
        with tempfile.TemporaryDirectory() as td:
            subprocess.run([sys.executable, os.path.abspath(__file__), "--config", args.config, "--write-pair0", td],
                           check=True, stdout=subprocess.DEVNULL)
            slcs = {k: np.load(os.path.join(td, k + ".npy")) for k in ("ref", "sec")}
        if args.samples == "ci16":  # the reference's pipe carries the widened samples
            from sentinel_gpu_processor_b200 import synth
            slcs = {k: torch.view_as_complex(synth.cint16(torch.from_numpy(v)).float()).numpy()
                    for k, v in slcs.items()}
        sc.dem = sc.ref_slc = sc.sec_slc = None
        if dev == "cuda":
            torch.cuda.empty_cache()
        sample = "burst pair 0 of the frame per step"
    else:
        base_sc = make_scene(args.config, 20261203 + 1000, "cpu")
        sc = refrun.make_reference_safe(base_sc)
        cfg = {"workload": f"burst pair {args.config}", "looks": [sc.rowlook, sc.collook],
               "goldstein": {"alpha": sc.alpha, "n_win": 32, "step": 8}, "parallelism": f"replicas{world}"}
        dem = sc.dem.numpy()
        slcs = {"ref": sc.ref_slc[0].numpy(), "sec": sc.sec_slc[0].numpy()}
        sample = "one burst pair per step"
    rl, cl = sc.rowlook, sc.collook
    L = sc.ref[0].radar.lines_per_burst
    S = sc.ref[0].radar.samples_per_burst
    wd = _workdir(dem.nbytes + 2 * slcs["ref"].nbytes)
    try:
        rscf, demf = refrun.write_dem(wd, sc.rsc, dem)
        dbs = {}
        for tag, acq in (("ref", sc.ref[0]), ("sec", sc.sec[0])):
            dbs[tag] = refrun.write_geo2rdr_inputs(wd, tag, acq, [slcs[tag]], rscf, demf)
        kb_inputs = None
        if os.path.exists(os.path.join(refrun.BIN, "kbench_chain")):
            kb_inputs = _kbench_inputs(wd, sc, dem, slcs)
        del dem, slcs

        def step():
            t0 = time.perf_counter()
            outs = {}
            for tag in ("ref", "sec"):
                o, _ = refrun.geo2rdr(dbs[tag], os.path.join(wd, tag), 1)
                outs[tag] = o[0]
            f1, f2 = os.path.join(wd, "ref_burst_0.gslc"), os.path.join(wd, "sec_burst_0.gslc")
            fo = os.path.join(wd, "pair.int")
            refrun.crossmul_daemon([(f1, f2, fo)], os.path.join(wd, "tasks.txt"), rl, cl, manual=False)
            ih, ifg = formats.read_raster(fo)
            # coherence: the reference's NumPy amplitude looks + coherence formula
            box = (int(ih[2]) * cl, int(ih[3]) * rl, int(ih[4]) * cl, int(ih[5]) * rl)
            (h1, d1), (h2, d2) = outs["ref"], outs["sec"]
            a1 = np.sqrt(oc.powlooks(ox.crop(h1, d1, box), rl, cl))
            a2 = np.sqrt(oc.powlooks(ox.crop(h2, d2, box), rl, cl))
            oc.coherence(ifg, a1, a2)
            gf = os.path.join(wd, "ifg.int")
            ifg.astype(np.complex64).tofile(gf)
            refrun.goldstein(gf, ifg.shape[0], ifg.shape[1], 32, sc.alpha)
            return time.perf_counter() - t0

        for _ in range(args.warmup):
            step()
        times = [step() for _ in range(args.steps)]
        kernel_only = None
        if kb_inputs is not None:
            ih, _ = formats.read_raster(os.path.join(wd, "pair.int"))
            try:
                kernel_only = _kbench_run(wd, kb_inputs, ih, (rl, cl), sc.alpha, L * S)
            except (RuntimeError, OSError, ValueError) as e:
                kernel_only = {"unavailable": f"kernel-only harness failed: {e}"[:300]}
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    mean = sum(times) / len(times)
    value = L * S / mean
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 geometry + c64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": f"{sample} (burst {L} x {S}, complex64): the reference executables geo2rdr x2, "
                                   "crossmul_daemon (its auto-tuned host workers), goldstein (sm_100a builds of the "
                                   "reference sources) + its NumPy coherence, wall clock, inputs in its file formats"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "world_size_requested": world,
        "repo_libraries_mapped": _repo_libraries_mapped(),
    }
    if kernel_only is not None:
        line["kernel_only"] = kernel_only
    print(json.dumps(line), flush=True)


ADJ_MARGIN = 16      # samples of the burst left out of the refinement grid on every side
ADJ_STEP_PX = 1e-3   # central-difference step of the offset parameters (samples)
ADJ_STEP_M = 0.4     # central-difference step along the height-error direction (metres)


def adjoint_measure(dev, steps, world, compact=False, n_bursts=8):
    """Adjoint of the coherence objective on ``n_bursts`` (8) bursts of 1500 x 21000: gradient
    evaluations per second through the fused adjoint, against central finite
    differences of every parameter plus one height-error direction run with
    the fused forward on the same GPU; a 50-step Adam refinement.  Returns a
    dict of the measurements (``compact``: no end-to-end or per-step details)."""
    import torch

    from sentinel_gpu_processor_b200 import synth
    from sentinel_gpu_processor_b200.refine import CoherenceObjective, CoregProblem, refine
    n = n_bursts
    # the reference grid is the burst's interior (16 samples off every edge):
    # no pixel's sinc support reaches the secondary burst's edge under the
    # perturbations, where J would jump as pixels enter or leave the support
    st = synth.make_refine_stack(n_bursts=n, config="c1", seed=20261203 + 3000, device=dev, margin=ADJ_MARGIN)
    pr = CoregProblem(st.sec_plans, st.ref, st.sec, st.az0, st.rg0, st.daz_dh, st.drg_dh, st.rowlook, st.collook)
    L, S = st.az0.shape[1:]
    params = torch.zeros((n, 6), dtype=torch.float32, device=dev)
    dh = torch.zeros((n, L, S), dtype=torch.float32, device=dev)
    gp = torch.empty_like(params)
    gh = torch.empty_like(dh)
    for _ in range(3):
        pr.gradient(params, dh, gp, gh)
        pr.objective(params, dh)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()

    def timed(fn, k):
        barrier(world)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(k):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(a.elapsed_time(b), world) / k

    t_adj = timed(lambda: pr.gradient(params, dh, gp, gh), steps)
    t_fwd = timed(lambda: pr.objective(params, dh), steps)
    # finite differences as one would run them: central differences of all
    # 6 n parameters and one height-error direction, forward evaluations only
    gd = torch.Generator(device=dev)
    gd.manual_seed(11)
    d = synth.gaussian_smooth(torch.randn((n, L, S), generator=gd, device=dev), 31.0)
    d = (d / d.std()).contiguous()
    # steps large enough that the float32 forward's rounding in J (~5e-11)
    # stays below 1e-3 of the difference, small enough for the truncation error
    step_p, step_h = ADJ_STEP_PX, ADJ_STEP_M
    fd = torch.zeros((n, 6), dtype=torch.float64, device=dev)
    fd_dir = torch.zeros(1, dtype=torch.float64, device=dev)

    def fd_gradient():
        for k in range(n):
            for j in range(6):
                p1 = params.clone()
                p1[k, j] += step_p
                jp = pr.objective(p1, dh).clone()
                p1[k, j] -= 2 * step_p
                fd[k, j] = (jp - pr.objective(p1, dh)) / (2 * step_p)
        jp = pr.objective(params, (dh + step_h * d).contiguous()).clone()
        fd_dir[0] = (jp - pr.objective(params, (dh - step_h * d).contiguous())) / (2 * step_h)

    t_fd = timed(fd_gradient, 1)
    pr.gradient(params, dh, gp, gh)
    adj_dir = float((gh.double() * d.double()).sum())
    rel_p = float((gp.double() - fd).norm() / fd.norm())
    rel_h = abs(adj_dir - float(fd_dir)) / abs(float(fd_dir))
    out = {"workload": f"{n} bursts of {L} x {S} complex64, offset polynomials (6 per burst, N(0, 0.05 px)) and a "
                       f"height-error field (10 m rms, 31-px Gaussian); looks {st.rowlook} x {st.collook}",
           "evals_per_s": 1e3 / t_adj, "gradient_ms": t_adj, "forward_ms": t_fwd,
           "finite_differences": {"evaluations": 12 * n + 2, "ms": t_fd, "speedup_adjoint_vs_fd": t_fd / t_adj,
                                  "step_px": step_p, "step_m": step_h,
                                  "rel_err_params_vs_gpu_fd": rel_p, "rel_err_height_direction_vs_gpu_fd": rel_h}}
    if not compact:
        # e2e: the public autograd API, pinned H2D of params and dh, D2H of both gradients
        ph, hh = params.cpu().pin_memory(), dh.cpu().pin_memory()
        gph, ghh = torch.empty_like(ph).pin_memory(), torch.empty_like(hh).pin_memory()

        def e2e_step():
            p_ = ph.to(dev, non_blocking=True).requires_grad_(True)
            h_ = hh.to(dev, non_blocking=True).requires_grad_(True)
            J = CoherenceObjective.apply(p_, h_, pr)
            J.backward()
            gph.copy_(p_.grad, non_blocking=True)
            ghh.copy_(h_.grad, non_blocking=True)

        e2e_step()
        t_e2e = timed(e2e_step, max(3, steps // 4))
        out["e2e"] = {"value": 1e3 / t_e2e, "unit": "evals/s", "h2d_bytes_per_step": (ph.numel() + hh.numel()) * 4,
                      "d2h_bytes_per_step": (gph.numel() + ghh.numel()) * 4}
    # refinement: 50 Adam steps from zero
    J0 = float(pr.objective(params, dh))
    a0, b0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    p_est, h_est, hist = refine(pr, steps=50, history=True)
    b0.record(stream)
    torch.cuda.synchronize()

    def offset_rms(p, h):
        xa = (torch.arange(L, device=dev)[:, None] - 0.5 * L) / L
        xr = (torch.arange(S, device=dev)[None, :] - 0.5 * S) / S
        dp = p - st.params_true
        e2 = 0.0
        for b in range(n):
            hb = h[b] - st.dh_true[b]
            ea = dp[b, 0] + dp[b, 1] * xa + dp[b, 2] * xr + st.daz_dh[b] * hb
            er = dp[b, 3] + dp[b, 4] * xa + dp[b, 5] * xr + st.drg_dh[b] * hb
            e2 += float((ea ** 2 + er ** 2).mean())
        return (e2 / n) ** 0.5

    out["refinement"] = {"adam_steps": 50, "ms": a0.elapsed_time(b0), "J_start": J0, "J_end": hist[-1],
                         "offset_rms_px_start": offset_rms(torch.zeros_like(p_est), torch.zeros_like(h_est)),
                         "offset_rms_px_end": offset_rms(p_est, h_est)}
    out["burst_px_per_s"] = n * L * S * 1e3 / t_adj
    out["achieved_gbs"] = 40.0 * n * L * S / (t_adj / 1e3) / 1e9
    del pr, st, params, dh, gp, gh, d
    torch.cuda.empty_cache()
    return out


STACK_SEED = 20261203 + 5000
STACK_BATCH = 10  # secondary dates per batch of the stack


def _mean_valid(coh):
    """Mean coherence over the interferogram's valid cells (coherence > 0:
    cells outside both bursts' overlap are 0)."""
    c = coh.float()
    v = c[c > 0]
    return float(v.mean()) if v.numel() else 0.0


def stack_measure(dev, steps, world, n_sec=29, offsets_rows=0, xmul=None):
    """The time series of one subswath: a reference date and ``n_sec``
    secondary dates of 9 bursts of 1500 x 21000 complex64 (baselines +-200 m,
    temporal coherence 0.9 exp(-dt / 60 d) at 12-day revisits, a 1 cm/yr
    deformation ramp).  Every reference-secondary burst pair runs through the
    batched frame path in batches of STACK_BATCH dates (one descriptor table
    and one CUDA graph per batch; the reference bursts stored once per batch);
    a batch's device time per replay is timed with CUDA events on resident
    inputs.  ``xmul``: crossmul fused into the geocoding (True), on geocoded
    windows (False: each burst geocoded once, the reference shared by the
    batch's pairs), or None to time both on the first batch and keep the
    faster.  ``offsets_rows`` > 0: for every burst pair, both bursts'
    geocoding sample coordinates against the float64 oracle on that many
    rows of the burst's DEM window (outside every timed region)."""
    import torch

    from sentinel_gpu_processor_b200 import synth
    from sentinel_gpu_processor_b200.chain import BatchedFrameChain
    st = synth.make_stack(seed=STACK_SEED, device=dev, n_sec=n_sec)
    nb = st.n_bursts
    ref_slcs = [synth.stack_slc(st, -1, b, dev) for b in range(nb)]
    batches = [list(range(i, min(i + STACK_BATCH, n_sec))) for i in range(0, n_sec, STACK_BATCH)]
    total_ms, px, per_pair, tried = 0.0, 0, [], {}
    for bi, dates in enumerate(batches):
        acqs = list(st.ref) + [st.sec[d][b] for d in dates for b in range(nb)]
        pairs = [(b, nb + j * nb + b) for j in range(len(dates)) for b in range(nb)]
        modes = [xmul] if xmul is not None else ([True, False] if bi == 0 else [tried["chosen"]])
        best = None
        for mode in modes:
            chain = BatchedFrameChain(acqs, None, st.rsc, st.rowlook, st.collook, st.alpha, device=dev, pairs=pairs,
                                      crossmul_fused=mode)
            for b in range(nb):
                chain.views[b].copy_(ref_slcs[b])
            for j, d in enumerate(dates):
                for b in range(nb):
                    chain.views[nb + j * nb + b].copy_(synth.stack_slc(st, d, b, dev))
            chain.capture(st.dem)
            ms = _timed_replays(chain.replay, steps)
            if bi == 0:
                tried["fused" if mode else "windows"] = ms
            if best is None or ms < best[0]:
                stats = []
                for k, r in enumerate(chain.results()):
                    d = dates[k // nb]
                    stats.append({"date": d, "burst": k % nb, "days": st.days[d],
                                  "baseline_m": round(st.baselines[d], 2), "coherence_sim": round(st.coherence[d], 4),
                                  "mean_coherence": None if r is None else _mean_valid(r.coh)})
                best = (ms, mode, chain.burst_pixels, stats)
            chain.graph = None
            del chain
            torch.cuda.empty_cache()
        ms, mode, bpx, stats = best
        tried["chosen"] = mode
        total_ms += ms
        px += bpx
        per_pair += stats
    out = {"workload": (f"time series of one subswath: 1 reference + {n_sec} secondary dates x {nb} bursts of "
                        f"{st.lines} x {st.samples} complex64 (band-limited speckle seen by every date at its own sample "
                        f"positions of the same ground points), 12-day revisits, baselines +-200 m, coherence "
                        f"0.9 exp(-dt/60 d), 1 cm/yr deformation ramp; batches of {STACK_BATCH} dates, one CUDA "
                        "graph per batch"),
           "value": px / (total_ms / 1e3), "unit": UNIT, "burst_pairs": len(per_pair), "burst_px": px,
           "ms_per_stack": total_ms, "batches": len(batches),
           "crossmul": "fused into the geocoding" if tried["chosen"] else "kernel on geocoded windows (reference "
                                                                       "bursts geocoded once per batch)",
           "first_batch_ms": {k: v for k, v in tried.items() if k != "chosen"}, "per_pair": per_pair}
    if offsets_rows > 0:
        import numpy as np

        from oracle import geo2rdr as og2
        from sentinel_gpu_processor_b200 import kernels, plan as _plan
        dem_h = st.dem.cpu().numpy()
        r = st.rsc

        def burst_stats(acq):
            """The geocoding's sample coordinates of one burst against the
            float64 oracle on ``offsets_rows`` rows of its DEM window."""
            pl = _plan.burst_plan(acq.radar, acq.orbit, acq.fm, acq.dc, acq.bursts[0], st.rsc)
            az, rg = kernels.geo2rdr_grid_offsets(pl, st.dem)
            # rows evenly inside the window (its edge rows can lie outside the burst)
            rows = np.linspace(0, pl.nrow - 1, offsets_rows + 2)[1:-1].round().astype(np.int64)
            rad = og2.Radar(**{k: getattr(acq.radar, k) for k in og2.Radar.__dataclass_fields__})
            b = og2.BurstMeta(**{k: getattr(acq.bursts[0], k) for k in og2.BurstMeta.__dataclass_fields__})
            oaz, org = og2.window_offsets(dem_h[pl.win_top:pl.win_bottom, pl.win_left:pl.win_right], rows, rad,
                                          acq.orbit, b, r.latmax + r.dlat * pl.win_top, r.lonmin + r.dlon * pl.win_left,
                                          r.dlat, r.dlon)
            gaz, grg = az.cpu().numpy()[rows], rg.cpu().numpy()[rows]
            used = ((org > b.first_valid_sample) & (org < b.last_valid_sample - 1) & (oaz >= b.first_valid_line + 5)
                    & (oaz < b.last_valid_line - 5))
            if not used.any():
                return {"max_az_px": 0.0, "max_rg_px": 0.0, "pixels": 0}
            return {"max_az_px": float(np.abs(gaz - oaz)[used].max()), "max_rg_px": float(np.abs(grg - org)[used].max()),
                    "pixels": int(used.sum())}

        ref_stats = [burst_stats(a) for a in st.ref]
        for e in per_pair:  # every reference-secondary burst pair: both bursts' sample coordinates
            s_ = burst_stats(st.sec[e["date"]][e["burst"]])
            q = ref_stats[e["burst"]]
            e["offset_err_px"] = {"ref": round(max(q["max_az_px"], q["max_rg_px"]), 10),
                                  "sec": round(max(s_["max_az_px"], s_["max_rg_px"]), 10),
                                  "pixels": q["pixels"] + s_["pixels"]}
            e["_sec"] = s_
        allst = ref_stats + [e.pop("_sec") for e in per_pair]
        out["offsets_vs_float64_oracle"] = {
            "bursts": len(allst), "rows_per_burst": offsets_rows, "pixels": sum(x["pixels"] for x in allst),
            "max_az_px": max(x["max_az_px"] for x in allst), "max_rg_px": max(x["max_rg_px"] for x in allst)}
        out["offset_px"] = max(out["offsets_vs_float64_oracle"]["max_az_px"],
                               out["offsets_vs_float64_oracle"]["max_rg_px"])
    return out


def run_stack(args):
    """configs C4 as its own bench line."""
    import torch
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    clocks = Clocks(local)
    clocks.start()
    m = stack_measure(dev, args.steps, world, offsets_rows=0 if (args.no_parity or world > 1) else 2)
    clk = clocks.stop()
    value = max_over_ranks(m["ms_per_stack"], world)
    line = {"metric": METRIC, "value": world * m["burst_px"] / (value / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": 3, "ms_per_step": value, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 geometry + c64", "data": "synthetic",
            "config": {"workload": m.pop("workload"), "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2"}, "stack": m}
    if clk is not None:
        line["clocks"] = clk
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_adjoint(args):
    """The adjoint measurement as its own bench line (metric: adjoint evals/s)."""
    import torch
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    clocks = Clocks(local)
    clocks.start()
    m = adjoint_measure(dev, args.steps, world, n_bursts=args.adjoint_bursts)
    clk = clocks.stop()
    line = {
        "metric": "adjoint evals/s (dJ/d offset polynomials and height field, J = -mean multilooked coherence)",
        "value": m["evals_per_s"], "unit": "evals/s", "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": m["gradient_ms"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 geometry and reductions)", "data": "synthetic",
        "config": {"workload": m["workload"] + "; fused resample -> crossmul -> multilook -> coherence -> gradient",
                   "l2": "inputs larger than L2", "parallelism": f"replicas{world}"},
        "forward_ms": m["forward_ms"], "burst_px_per_s": m["burst_px_per_s"],
        "finite_differences": m["finite_differences"], "refinement": m["refinement"], "e2e": m["e2e"],
        "gpu_launches": 3 * args.steps,
        "roofline": {"bound": "hbm", "kernel": "adjoint_kernel<grad>", "achieved": m["achieved_gbs"], "unit": "GB/s",
                     "limiter": "FP32 taps: 3 interpolations x 64 complex x real FMA per pixel; HBM bytes 40 B/px"},
    }
    if clk is not None:
        line["clocks"] = clk
    if rank == 0:
        print(json.dumps(line))


def main():
    args = parse()
    if args.write_pair0:
        write_pair0(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "adjoint":
        run_adjoint(args)
    elif args.config == "stack":
        run_stack(args)
    else:
        run_s1b(args)


if __name__ == "__main__":
    main()
