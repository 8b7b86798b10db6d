"""Benchmark: IW-burst pixels/s of the chain geo2rdr -> resample -> ifg -> coherence -> Goldstein.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl s1b|reference] [--config c1]

A step is one pass of the chain over one reference/secondary burst pair of
one full IW burst (1500 lines x 21000 samples, complex64, looks 4 x 20,
Goldstein alpha 0.6, 32 x 32 patches): TOPS deramp and FP64 geocoding of
both SLCs onto the DEM grid, crossmul + multilook + amplitude looks +
coherence, Goldstein filter.  ``value`` = burst pixels (lines x samples of
the reference burst, counted once per pair) per second with inputs resident
in HBM; ``e2e`` = the same through the host-buffer call
(``chain.process_pair_host``) with H2D of both SLCs and the DEM and D2H of
the products inside the timed region.

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
# DRAM bytes of one geocoding launch per geo pixel, from the ncu capture
# summarised in profiles/geo2rdr_c1.md (dram__bytes_read.sum + write.sum).
GEO_DRAM_BYTES_PER_GEO_PX = None


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="s1b", choices=["s1b", "reference"])
    ap.add_argument("--config", default="c1", choices=["c1", "c0", "small"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
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
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                      "-i", str(self.index), "-lms", "200"], stdout=open(self.path, "w"),
                                     stderr=subprocess.DEVNULL)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx = float(p[2])
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def make_scene(config, seed, device):
    from sentinel_gpu_processor_b200 import synth
    return synth.make_pair(config, seed=seed, device=device)


# ----------------------------------------------------------------------------
# CPU baseline: the float64 oracle on a bounded sample of the same workload
# ----------------------------------------------------------------------------

def cpu_baseline():
    import numpy as np

    from oracle import coherence as oc
    from oracle import crossmul as ox
    from oracle import geo2rdr as og2
    from oracle import goldstein as ogs
    from sentinel_gpu_processor_b200 import synth
    sc = synth.make_pair("small", seed=99)  # 160 x 640 burst, same geometry and processing
    rsc = og2.Rsc(**sc.rsc.__dict__)
    times = []
    for _ in range(2):
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
        times.append(time.perf_counter() - t0)
    dt = min(times)
    px = sc.burst_pixels
    return {"value": px / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"float64 NumPy oracle chain on a 160 x 640 burst pair of the same geometry and processing "
                      f"({px} burst px, best of 2 runs, {dt:.2f} s)"}


# ----------------------------------------------------------------------------
# s1b arm
# ----------------------------------------------------------------------------

def run_s1b(args):
    import torch

    from sentinel_gpu_processor_b200.chain import PairChain, process_pair_host
    rank, world, local = dist_setup(args.gpus)
    dev = torch.device("cuda", local)
    seed = 20261203 + 1000 * 1 + rank
    sc = make_scene(args.config, seed, dev)
    chain = PairChain(sc.ref[0], sc.sec[0], sc.rsc, sc.rowlook, sc.collook, sc.alpha, device=dev)
    ref, sec, dem = sc.ref_slc[0], sc.sec_slc[0], sc.dem
    p0 = chain.plans[0]
    geo_px = [p.nrow * p.ncol for p in chain.plans]
    res = None
    for _ in range(max(args.warmup, 3)):
        res = chain.run(ref, sec, dem)
    torch.cuda.synchronize()
    if res is None:
        raise SystemExit("empty interferogram for the synthetic pair")
    stream = torch.cuda.current_stream()
    # kernel events around the two geocoding launches of every timed step
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(2 * args.steps)]
    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    from sentinel_gpu_processor_b200 import kernels
    for k in range(args.steps):
        for i, (pl, slc) in enumerate(zip(chain.plans, (ref, sec))):
            kernels.deramp(pl, slc.reshape(-1), out=chain.deramped[i])
            e0, e1 = ev[2 * k + i]
            e0.record(stream)
            kernels.geo2rdr(pl, dem, chain.deramped[i], out=chain.geo[i], rows=chain.rows[2 * i:2 * i + 2])
            e1.record(stream)
        hs = chain.headers()
        res = chain.interfere(hs)
    stop.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    elapsed_ms = start.elapsed_time(stop)
    elapsed_ms = max_over_ranks(elapsed_ms, world)
    geo_ms = [a.elapsed_time(b) for a, b in ev]
    geo_avg_ms = sum(geo_ms) / len(geo_ms)
    value = world * args.steps * chain.burst_pixels / (elapsed_ms / 1e3)

    # end to end through the host-buffer call
    ref_h = ref.cpu().pin_memory()
    sec_h = sec.cpu().pin_memory()
    dem_h = dem.cpu().pin_memory()
    dev_in, host_out = None, None
    dev_in = {"ref": torch.empty_like(ref), "sec": torch.empty_like(sec), "dem": torch.empty_like(dem)}
    _, host_out, _, _ = process_pair_host(chain, ref_h, sec_h, dem_h, dev_in, host_out)
    k_e2e = max(3, args.steps // 2)
    barrier(world)
    torch.cuda.synchronize()
    s2, t2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(k_e2e):
        _, host_out, h2d, d2h = process_pair_host(chain, ref_h, sec_h, dem_h, dev_in, host_out)
    t2.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(s2.elapsed_time(t2), world)
    e2e = world * k_e2e * chain.burst_pixels / (e2e_ms / 1e3)

    peak, peak_kind = peaks()
    geo_bytes = GEO_BYTES_PER_GEO_PX * (geo_px[0] + geo_px[1]) / 2 + GEO_BYTES_PER_BURST_PX * chain.burst_pixels
    achieved = geo_bytes / (geo_avg_ms / 1e3) / 1e9
    traffic = None
    if GEO_DRAM_BYTES_PER_GEO_PX is not None:
        traffic = GEO_DRAM_BYTES_PER_GEO_PX * (geo_px[0] + geo_px[1]) / 2
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": elapsed_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 geometry + c64", "data": "synthetic",
        "config": {"workload": f"one IW burst pair {p0.lines} x {p0.samples} complex64 (configs[1])",
                   "lines": p0.lines, "samples": p0.samples, "looks": [sc.rowlook, sc.collook],
                   "goldstein": {"alpha": sc.alpha, "n_win": 32, "step": 8},
                   "geo_px": geo_px, "ifg_ml": list(res.ifg.shape),
                   "l2": "inputs larger than L2 (two 252 MB SLCs + DEM per step)", "parallelism": f"replicas{world}"},
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": PairChain.launches_per_step() * args.steps,
        "roofline": {"bound": "hbm", "kernel": "geo2rdr_kernel", "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": peak_kind, "bytes_per_launch": geo_bytes, "launch_ms": geo_avg_ms,
                     "note": "geocoding is FP64-compute bound (zero-Doppler Newton); its HBM fraction is low "
                             "by design"},
        "kernels_ms": {"geo2rdr_avg": geo_avg_ms, "step": elapsed_ms / args.steps},
    }
    if clk is not None:
        line["clocks"] = clk
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# ----------------------------------------------------------------------------
# reference arm
# ----------------------------------------------------------------------------

def run_reference(args):
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
    # the reference geo2rdr overruns its DEM/output buffers on some grids
    # (oracle/refrun.geo2rdr_buffers_safe); run it only on a checked-safe grid
    sc = refrun.make_reference_safe(make_scene(args.config, 20261203 + 1000, "cpu"))
    base = "/dev/shm" if os.path.isdir("/dev/shm") else None
    wd = tempfile.mkdtemp(prefix="s1b_refbench_", dir=base)
    try:
        rscf, demf = refrun.write_dem(wd, sc.rsc, sc.dem.numpy())
        dbs = {}
        for tag, acq, slc in (("ref", sc.ref[0], sc.ref_slc[0]), ("sec", sc.sec[0], sc.sec_slc[0])):
            dbs[tag] = refrun.write_geo2rdr_inputs(wd, tag, acq, [slc.numpy()], rscf, demf)
        L = sc.ref[0].radar.lines_per_burst
        S = sc.ref[0].radar.samples_per_burst

        def step():
            t0 = time.perf_counter()
            outs = {}
            for tag in ("ref", "sec"):
                o, _ = refrun.geo2rdr(dbs[tag], os.path.join(wd, tag), 1)
                outs[tag] = o[0]
            f1, f2 = os.path.join(wd, "ref_burst_0.gslc"), os.path.join(wd, "sec_burst_0.gslc")
            fo = os.path.join(wd, "pair.int")
            refrun.crossmul_daemon([(f1, f2, fo)], os.path.join(wd, "tasks.txt"), sc.rowlook, sc.collook,
                                   manual=False)
            ih, ifg = formats.read_raster(fo)
            # coherence: the reference's NumPy amplitude looks + coherence formula
            box = (int(ih[2]) * sc.collook, int(ih[3]) * sc.rowlook, int(ih[4]) * sc.collook, int(ih[5]) * sc.rowlook)
            (h1, d1), (h2, d2) = outs["ref"], outs["sec"]
            a1 = np.sqrt(oc.powlooks(ox.crop(h1, d1, box), sc.rowlook, sc.collook))
            a2 = np.sqrt(oc.powlooks(ox.crop(h2, d2, box), sc.rowlook, sc.collook))
            oc.coherence(ifg, a1, a2)
            gf = os.path.join(wd, "ifg.int")
            ifg.astype(np.complex64).tofile(gf)
            refrun.goldstein(gf, ifg.shape[0], ifg.shape[1], 32, sc.alpha)
            return time.perf_counter() - t0

        for _ in range(args.warmup):
            step()
        times = [step() for _ in range(args.steps)]
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    mean = sum(times) / len(times)
    value = L * S / mean
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": mean * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 geometry + c64", "data": "synthetic",
        "config": {"workload": f"one IW burst pair {L} x {S} complex64 (configs[1])", "lines": L, "samples": S,
                   "looks": [sc.rowlook, sc.collook], "goldstein": {"alpha": sc.alpha, "n_win": 32, "step": 8},
                   "files": "reference formats on /dev/shm"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "sample": "the reference executables geo2rdr x2, crossmul_daemon, goldstein (sm_100a "
                                   "builds of the reference sources) + its NumPy coherence, per burst pair"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "world_size_requested": world,
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_s1b(args)


if __name__ == "__main__":
    main()
