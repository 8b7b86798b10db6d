"""The command-line drop-ins run on the golden fixture's inputs, written in
the reference's file formats (parameter DB, orbit/FM/DC text, RSC, DEM, raw
SLC), against the outputs the reference executables produced from the same
files (tests/golden/ref_chain_tiny.npz): .gslc crops and data, the
interferogram raster and header, the Goldstein output, stdout lines and exit
codes."""
import io
import os

import numpy as np
import pytest

from helpers import GOLD, golden_acq, golden_rsc, phase_rms, rel_err
from oracle import refrun
from sentinel_gpu_processor_b200 import cli, formats

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def z():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def files(z, tmp_path_factory, cuda):
    wd = str(tmp_path_factory.mktemp("cli"))
    rscf, demf = refrun.write_dem(wd, golden_rsc(z), z["dem"])
    dbs = {}
    for tag in ("ref", "sec"):
        dbs[tag] = refrun.write_geo2rdr_inputs(wd, tag, golden_acq(z, tag + "_"), [z[tag + "_slc"]], rscf, demf)
    return wd, dbs


def _check_gslc(path, z, tag):
    h, d = formats.read_raster(path)
    gh, gd = z[tag + "_gslc_header"], z[tag + "_gslc"]
    np.testing.assert_array_equal(np.asarray(h)[[0, 1, 2, 4]], np.asarray(gh)[[0, 1, 2, 4]])
    # the reference's racy row reduction can only drop rows: our crop contains its crop
    assert int(h[3]) <= int(gh[3]) and int(h[5]) >= int(gh[5])
    ours = d[int(gh[3]) - int(h[3]):int(gh[5]) - int(h[3])]
    m = (np.abs(ours) > 0) & (np.abs(gd) > 0)
    assert ((np.abs(ours) > 0) != (np.abs(gd) > 0)).mean() < 1e-3
    assert phase_rms(ours, gd, m) < 1e-3


@pytest.mark.parametrize("mode", ["file", "stdin"])
def test_geo2rdr_dropin(z, files, mode):
    wd, dbs = files
    for tag in ("ref", "sec"):
        out = os.path.join(wd, f"{mode}_{tag}")
        if mode == "file":
            rc = cli.geo2rdr_main(["geo2rdr", dbs[tag], out])
        else:
            rc = cli.geo2rdr_main(["geo2rdr", dbs[tag], out, "--stdin"],
                                  stdin=io.BytesIO(np.ascontiguousarray(z[tag + "_slc"]).tobytes()))
        assert rc == 0
        _check_gslc(out + "_burst_0.gslc", z, tag)


def test_geo2rdr_stdin_short_read_fails(z, files):
    wd, dbs = files
    rc = cli.geo2rdr_main(["geo2rdr", dbs["ref"], os.path.join(wd, "short"), "--stdin"], stdin=io.BytesIO(b"\0" * 64))
    assert rc == 1


def test_crossmul_daemon_dropin(z, files):
    """On the .gslc files the reference geo2rdr wrote: identical headers."""
    wd, dbs = files
    for tag in ("ref", "sec"):
        formats.write_raster(os.path.join(wd, f"d_{tag}_burst_0.gslc"), z[tag + "_gslc_header"], z[tag + "_gslc"])
    rl, cl = (int(v) for v in z["looks"])
    tasks = os.path.join(wd, "tasks.txt")
    out = os.path.join(wd, "pair.int")
    outf = os.path.join(wd, "pair_phase.int")
    with open(tasks, "w") as f:
        f.write(f"{wd}/d_ref_burst_0.gslc {wd}/d_sec_burst_0.gslc {out}\n")
    lines = []
    rc = cli.crossmul_daemon_main(["crossmul_daemon", "--rowlook", str(rl), "--collook", str(cl), "--tasks-file",
                                   tasks], emit=lines.append)
    assert rc == 0
    assert lines[0] == f"OK {out}" and lines[-1].startswith("SUMMARY 1 0 1 ")
    h, ifg = formats.read_raster(out)
    np.testing.assert_array_equal(np.asarray(h)[:6], z["ifg_header"][:6])
    assert phase_rms(ifg, z["ifg"], np.abs(z["ifg"]) > 0) < 1e-3
    assert rel_err(ifg, z["ifg"]) < 1e-3
    with open(tasks, "w") as f:
        f.write(f"{wd}/d_ref_burst_0.gslc {wd}/d_sec_burst_0.gslc {outf}\n")
    assert cli.crossmul_daemon_main(["crossmul_daemon", "--rowlook", str(rl), "--collook", str(cl), "--out-float",
                                     "--tasks-file", tasks], emit=lines.append) == 0
    hp, ph = formats.read_raster(outf, dtype=np.float32)
    np.testing.assert_array_equal(np.asarray(hp)[:6], z["phase_header"][:6])
    d = np.angle(np.exp(1j * (ph.astype(np.float64) - z["phase"])))
    assert np.sqrt(np.mean(d ** 2)) < 1e-3
    # a missing input fails that task only, with exit code 1
    with open(tasks, "w") as f:
        f.write(f"{wd}/missing.gslc {wd}/d_sec_burst_0.gslc {out}\n")
    lines = []
    assert cli.crossmul_daemon_main(["crossmul_daemon", "--tasks-file", tasks], emit=lines.append) == 1
    assert lines[-1].startswith("SUMMARY 0 1 1 ")


def test_goldstein_dropin(z, files, capsys):
    wd, _ = files
    n_win, alpha = int(z["gold_params"][0]), float(z["gold_params"][1])
    nrow, ncol = z["gold_in"].shape
    src = os.path.join(wd, "g1.bin")
    z["gold_in"].astype(np.complex64).tofile(src)
    lst = os.path.join(wd, "list.txt")
    with open(lst, "w") as f:
        f.write(src + "\n")
    assert cli.goldstein_main(["goldstein", lst, str(nrow), str(ncol), str(n_win), str(alpha)]) == 0
    assert f"Run Goldstein filter, input: {src}, output: {src}.filt" in capsys.readouterr().out
    got = np.fromfile(src + ".filt", dtype=np.complex64).reshape(nrow, ncol)
    want = z["gold_out"]
    assert phase_rms(got, want, np.abs(want) > 0) < 1e-3
    assert rel_err(got, want) < 1e-4


def test_chained_geo2rdr_and_daemon(z, files):
    """Our geo2rdr then our daemon: the reference's racy crop can drop edge
    rows, so our interferogram box contains its box; overlapping rows agree."""
    wd, dbs = files
    for tag in ("ref", "sec"):
        assert cli.geo2rdr_main(["geo2rdr", dbs[tag], os.path.join(wd, "c_" + tag)]) == 0
    rl, cl = (int(v) for v in z["looks"])
    tasks = os.path.join(wd, "tasks_c.txt")
    out = os.path.join(wd, "chain.int")
    with open(tasks, "w") as f:
        f.write(f"{wd}/c_ref_burst_0.gslc {wd}/c_sec_burst_0.gslc {out}\n")
    assert cli.crossmul_daemon_main(["crossmul_daemon", "--rowlook", str(rl), "--collook", str(cl), "--tasks-file",
                                     tasks], emit=lambda s: None) == 0
    h, ifg = formats.read_raster(out)
    gh, g = z["ifg_header"], z["ifg"]
    np.testing.assert_array_equal(np.asarray(h)[[0, 1, 2, 4]], np.asarray(gh)[[0, 1, 2, 4]])
    assert int(h[3]) <= int(gh[3]) and int(h[5]) >= int(gh[5])
    ours = ifg[int(gh[3]) - int(h[3]):int(gh[5]) - int(h[3])]
    assert phase_rms(ours, g, np.abs(g) > 0) < 1e-3
