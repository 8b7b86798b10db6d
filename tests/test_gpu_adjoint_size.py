"""The adjoint at the differentiation workload's size: 8 bursts of 1500 x
21000 (the refinement grid is each burst's interior, 16 samples off every
edge, so no pixel's 8 x 8 sinc support reaches the secondary burst's edge,
where the objective would jump as pixels enter or leave the support).

The gradient of the fused adjoint is checked against central finite
differences of the same float32 forward on the GPU: every offset-polynomial
parameter (step 1e-3 samples) and one smoothed height-error direction (step
0.4 m; the forward's rounding in J is ~5e-11, so smaller steps measure
rounding).  The float64 oracle checks the same gradient at a small size
(test_gpu_adjoint.py).  Bound (north star): relative error <= 1e-3; and the
adjoint is at least 20 times faster than the finite differences.
"""
import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402

pytestmark = pytest.mark.gpu


def test_adjoint_matches_gpu_finite_differences_at_size(cuda):
    m = bench.adjoint_measure(cuda, 3, 1, compact=True)
    fd = m["finite_differences"]
    assert fd["rel_err_params_vs_gpu_fd"] <= 1e-3, fd
    assert fd["rel_err_height_direction_vs_gpu_fd"] <= 1e-3, fd
    assert fd["speedup_adjoint_vs_fd"] >= 20, fd
    assert m["refinement"]["offset_rms_px_end"] < 0.25 * m["refinement"]["offset_rms_px_start"]
