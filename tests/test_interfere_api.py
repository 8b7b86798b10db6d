"""s1proc's interfere() call surface (s1proc/interfere.py:17-78, 536-704):
burst matching per subswath, burst-pair file names, the all-or-nothing
tuning contract.  Host logic only (no GPU)."""
import os

import numpy as np
import pytest

from sentinel_gpu_processor_b200 import interfere as I


def _gslc(path, box, nrow0=400, ncol0=500):
    h = np.zeros(64, dtype=np.int32)
    h[:6] = [nrow0, ncol0, *box]
    with open(path, "wb") as f:
        h.tofile(f)
        np.zeros((box[3] - box[1]) * (box[2] - box[0]), dtype=np.complex64).tofile(f)
    return path


def test_burst_pair_tasks_match_nearest_rows_per_subswath(tmp_path):
    d = str(tmp_path)
    ref = [_gslc(os.path.join(d, f"20200101_S1A_AAAA_iw1_burst_{i}.gslc"), (10, 100 * i, 200, 100 * i + 120))
           for i in range(3)]
    ref += [_gslc(os.path.join(d, "20200101_S1A_AAAA_iw2_burst_0.gslc"), (190, 5, 400, 130))]
    # the secondary's bursts are listed out of order and shifted by a few rows
    sec = [_gslc(os.path.join(d, f"20200113_S1B_BBBB_iw1_burst_{i}.gslc"), (12, 100 * i + 3, 201, 100 * i + 118))
           for i in (2, 0, 1)]
    tasks = I.burst_pair_tasks(ref, sec, "igrams")
    assert len(tasks) == 3  # iw2 has no secondary burst: no pair
    for k, (f1, f2, out) in enumerate(tasks):
        assert f1.endswith(f"iw1_burst_{k}.gslc") and f2.endswith(f"iw1_burst_{k}.gslc")
        assert out == os.path.join("igrams", f"20200101_S1A_AAAA_iw1_burst_{k}_20200113_S1B_BBBB_iw1_burst_{k}.int")


def test_tuning_contract():
    I.check_tuning()
    I.check_tuning(1, 2, 1, 4, 8)
    for bad in ((1, -1, -1, -1, -1), (0, 1, 1, 1, 1), (1, 1, 1, 1, 2.0)):
        with pytest.raises(SystemExit) as e:
            I.check_tuning(*bad)
        assert e.value.code == 1
