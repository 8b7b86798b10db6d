"""Goldstein filter parity on the GPU against the oracle (oracle/goldstein.py,
float64 NumPy FFT standing in for cuFFT).

Tolerance: RMS wrapped-phase difference <= 1e-3 rad (north star) and a
relative amplitude bound; the float32 FFT of the kernel differs from a
float64 FFT by ~1e-6 relative.
"""
import numpy as np
import pytest
import torch

from helpers import phase_rms, rel_err
from oracle import goldstein as og
from sentinel_gpu_processor_b200 import _lib, kernels

pytestmark = pytest.mark.gpu


def _ifg(rng, nrow, ncol, noise=0.6):
    y, x = np.mgrid[0:nrow, 0:ncol]
    ph = 0.09 * x + 0.05 * y + 2.0 * np.sin(x / 17.0) * np.cos(y / 23.0)
    z = np.exp(1j * ph) + noise * (rng.standard_normal((nrow, ncol)) + 1j * rng.standard_normal((nrow, ncol)))
    return z.astype(np.complex64)


@pytest.mark.parametrize("shape,alpha", [((32, 32), 0.5), ((64, 96), 0.5), ((75, 133), 0.6), ((120, 250), 0.8)])
def test_goldstein_matches_oracle(cuda, shape, alpha):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    img = _ifg(rng, *shape)
    got = kernels.goldstein(torch.from_numpy(img).to(cuda), alpha).cpu().numpy()
    want = og.goldstein(img, 32, alpha)
    m = np.abs(want) > 1e-3 * np.abs(want).max()
    assert phase_rms(got, want, m) < 1e-3
    assert rel_err(got, want) < 2e-5


def test_goldstein_alpha_zero_and_zeros(cuda):
    rng = np.random.default_rng(2)
    img = _ifg(rng, 48, 64)
    got = kernels.goldstein(torch.from_numpy(img).to(cuda), 0.0).cpu().numpy()
    want = og.goldstein(img, 32, 0.0)
    assert rel_err(got, want) < 2e-5
    z = torch.zeros((40, 40), dtype=torch.complex64, device=cuda)
    assert torch.count_nonzero(kernels.goldstein(z, 0.5)) == 0


def test_goldstein_deterministic_and_inplace(cuda):
    rng = np.random.default_rng(3)
    img = torch.from_numpy(_ifg(rng, 80, 120)).to(cuda)
    a = kernels.goldstein(img, 0.5)
    b = kernels.goldstein(img, 0.5)
    assert torch.equal(a, b)
    c = img.clone()
    kernels.goldstein(c, 0.5, out=c)  # reads finish before the gather writes
    assert torch.equal(a, c)


def test_goldstein_rejects_bad_sizes(cuda):
    with pytest.raises(_lib.S1BError):
        kernels.goldstein(torch.zeros((20, 64), dtype=torch.complex64, device=cuda), 0.5)
    with pytest.raises(_lib.S1BError):
        kernels.goldstein(torch.zeros((64, 64), dtype=torch.complex64, device=cuda), 0.5, n_win=16)
