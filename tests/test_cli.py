"""The command-line drop-ins (sentinel_gpu_processor_b200/cli.py, bin/):
usage lines, argument validation and exit codes of the reference
executables (geo2rdr.cu:704-734, crossmul_daemon.cu:1744-1911,
crossmul.cu:285-298, goldstein.cu:504-524), without a GPU."""
import os
import subprocess
import sys

from sentinel_gpu_processor_b200 import cli

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "sentinel_gpu_processor_b200", "bin")


def test_usage_lines_exit_zero(capsys):
    assert cli.geo2rdr_main(["geo2rdr"]) == 0
    assert cli.crossmul_main(["crossmul", "a"]) == 0
    assert cli.goldstein_main(["goldstein", "a", "1", "2"]) == 0
    out = capsys.readouterr().out
    assert "Usage: geo2rdr dbname slcoutfile [slcinfile] [--stdin] [--gpu DEVICE_ID]" in out
    assert "Usage: crossmul input_file rowlook collook out_float" in out
    assert "Usage: goldstein in_str nrow ncol n_win alpha [out_str]" in out


def test_gpu_argument_anywhere():
    assert cli._gpu_arg(["x", "a", "--gpu", "3", "b"]) == 3
    assert cli._gpu_arg(["x", "-g", "1"]) == 1
    assert cli._gpu_arg(["x", "a", "--gpu"]) == -1


def test_daemon_argument_checks(tmp_path, capsys):
    # partial tuning overrides are rejected
    assert cli.crossmul_daemon_main(["d", "--tasks-file", "t", "--io-workers", "2"]) == 1
    assert "Partial overrides are not allowed" in capsys.readouterr().err
    assert cli.crossmul_daemon_main(["d", "--rowlook", "2"]) == 1
    assert "--tasks-file <path> is required" in capsys.readouterr().err
    empty = tmp_path / "tasks.txt"
    empty.write_text("\n\n")
    assert cli.crossmul_daemon_main(["d", "--tasks-file", str(empty)]) == 0
    assert "No tasks found" in capsys.readouterr().err
    bad = tmp_path / "bad.txt"
    bad.write_text("only two\n\n")
    assert cli.read_tasks(str(bad)) == []
    assert "skipping malformed task line" in capsys.readouterr().err


def test_goldstein_inputs(tmp_path, capsys):
    lst = tmp_path / "list"
    lst.write_text("a.bin\nb.bin\n")
    assert cli.goldstein_inputs(str(lst)) == (["a.bin", "b.bin"], False)
    assert cli.goldstein_inputs("x.int") == (["x.int"], True)
    assert cli.goldstein_main(["g", str(tmp_path / "missing"), "4", "4", "32", "0.5"]) == 0
    assert "Input list is empty, nothing to filter." in capsys.readouterr().out


def test_bin_stubs_run():
    for name in ("geo2rdr", "crossmul_daemon", "crossmul", "goldstein"):
        path = os.path.join(BIN, name)
        assert os.access(path, os.X_OK)
    r = subprocess.run([sys.executable, os.path.join(BIN, "geo2rdr")], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.startswith("Usage: geo2rdr")
