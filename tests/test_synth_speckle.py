"""Band-limited speckle of the stack workload: unit power, no spectral
content outside the kept band, and values between samples fixed by the
samples (a half-sample shift by FFT interpolation stays highly correlated
with the field sampled there)."""
import math

import numpy as np
import torch

from sentinel_gpu_processor_b200 import synth


def test_band_limited_speckle_power_and_band():
    gen = torch.Generator()
    gen.manual_seed(5)
    z = synth.band_limited_speckle(256, 512, gen, "cpu", band=0.8).numpy().astype(np.complex128)
    assert z.shape == (256, 512)
    assert abs(np.mean(np.abs(z) ** 2) - 1.0) < 0.05
    f = np.fft.fft2(z)
    fa = np.abs(np.fft.fftfreq(256)) > 0.4
    fr = np.abs(np.fft.fftfreq(512)) > 0.4
    outside = np.abs(f[fa, :]).max(), np.abs(f[:, fr]).max()
    assert max(outside) < 1e-3 * np.abs(f).max()


def test_band_limited_speckle_is_smooth_between_samples():
    gen = torch.Generator()
    gen.manual_seed(9)
    z = synth.band_limited_speckle(128, 1024, gen, "cpu", band=0.8).numpy().astype(np.complex128)
    # exact half-sample shift in range of a band-limited field (FFT phase ramp)
    k = np.fft.fftfreq(1024)
    zs = np.fft.ifft(np.fft.fft(z, axis=1) * np.exp(2j * math.pi * k * 0.5)[None, :], axis=1)
    # linear interpolation of the samples predicts the shifted field well
    lin = 0.5 * (z + np.roll(z, -1, axis=1))
    c = np.abs(np.vdot(lin, zs)) / np.sqrt(np.vdot(lin, lin).real * np.vdot(zs, zs).real)
    assert c > 0.85
