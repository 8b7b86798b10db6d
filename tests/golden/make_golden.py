"""Generate ``ref_chain_tiny.npz``: inputs and outputs of the reference CUDA
executables (geo2rdr, crossmul_daemon, goldstein) on a seeded tiny scene.

Needs a CUDA GPU and the executables built by ``oracle/build_ref.py``.
Run from the repository root: ``python tests/golden/make_golden.py [out.npz]``.
The fixture pins the oracle restatement (tests/test_golden_chain.py, CPU) and
the s1b kernels (same file, GPU tests) to the reference without rebuilding it.
"""
import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import refrun  # noqa: E402
from sentinel_gpu_processor_b200 import formats, synth  # noqa: E402

SEED = 424242
N_WIN = 32


def main(out=None):
    out = out or os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_chain_tiny.npz")
    sc = synth.make_pair("tiny", seed=SEED)
    wd = tempfile.mkdtemp(prefix="s1b_golden_")
    rscf, demf = refrun.write_dem(wd, sc.rsc, sc.dem.numpy())
    res = {}
    for tag, acq, slc in (("ref", sc.ref[0], sc.ref_slc[0]), ("sec", sc.sec[0], sc.sec_slc[0])):
        db = refrun.write_geo2rdr_inputs(wd, tag, acq, [slc.numpy()], rscf, demf)
        outs, _ = refrun.geo2rdr(db, os.path.join(wd, tag), 1)
        if outs[0] is None:
            raise SystemExit(f"reference geo2rdr produced no output for {tag}")
        res[tag] = outs[0]
    f1, f2 = os.path.join(wd, "ref_burst_0.gslc"), os.path.join(wd, "sec_burst_0.gslc")
    fo = os.path.join(wd, "pair.int")
    refrun.crossmul_daemon([(f1, f2, fo)], os.path.join(wd, "tasks.txt"), sc.rowlook, sc.collook)
    ih, ifg = formats.read_raster(fo)
    fo2 = os.path.join(wd, "pair_phase.int")
    refrun.crossmul_daemon([(f1, f2, fo2)], os.path.join(wd, "tasks2.txt"), sc.rowlook, sc.collook, out_float=True)
    ph_h, phase = formats.read_raster(fo2, dtype=np.float32)
    # Goldstein on a smooth-fringe image of the size class of a multilooked burst
    rng = np.random.default_rng(SEED)
    nrow, ncol = 72, 136
    y, x = np.mgrid[0:nrow, 0:ncol]
    gin = (np.exp(1j * (0.11 * x + 0.04 * y)) + 0.6 * (rng.standard_normal((nrow, ncol)) +
                                                       1j * rng.standard_normal((nrow, ncol)))).astype(np.complex64)
    gf = os.path.join(wd, "g.int")
    gin.tofile(gf)
    gout, _ = refrun.goldstein(gf, nrow, ncol, N_WIN, sc.alpha)
    acq_r, acq_s = sc.ref[0], sc.sec[0]

    def acq_arrays(prefix, acq):
        r = acq.radar
        b = acq.bursts[0]
        return {
            prefix + "radar": np.array([r.samples_per_burst, r.lines_per_burst, r.prf, r.wvl, r.hmin, r.hmax,
                                        r.range_sampling_rate, r.slant_range_time, r.azimuth_steering_rate,
                                        r.azimuth_time_interval, r.radar_frequency]),
            prefix + "burst": np.array([b.azimuth_time, b.first_valid_line, b.last_valid_line,
                                        b.first_valid_sample, b.last_valid_sample]),
            prefix + "tt": acq.orbit[0], prefix + "xx": acq.orbit[1], prefix + "vv": acq.orbit[2],
            prefix + "fm": acq.fm, prefix + "dc": acq.dc,
        }

    arrays = {}
    arrays.update(acq_arrays("ref_", acq_r))
    arrays.update(acq_arrays("sec_", acq_s))
    rsc = sc.rsc
    np.savez_compressed(
        out, seed=SEED, rsc=np.array([rsc.nlat, rsc.nlon, rsc.latmax, rsc.lonmin, rsc.dlat, rsc.dlon]),
        dem=sc.dem.numpy(), ref_slc=sc.ref_slc[0].numpy(), sec_slc=sc.sec_slc[0].numpy(),
        ref_gslc_header=res["ref"][0], ref_gslc=res["ref"][1], sec_gslc_header=res["sec"][0],
        sec_gslc=res["sec"][1], looks=np.array([sc.rowlook, sc.collook]), ifg_header=ih, ifg=ifg,
        phase_header=ph_h, phase=phase, gold_in=gin, gold_out=gout, gold_params=np.array([N_WIN, sc.alpha]),
        **arrays)
    print("wrote", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else None)
