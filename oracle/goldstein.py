"""Oracle of the reference Goldstein filter (``goldstein`` executable).

Test infrastructure only (see ``oracle/__init__.py``).

Follows ``csrc/src/goldstein.cu``:
  * 43-52    7x7 smoothing table (the reference project's constants)
  * 87-123   gaussian_filter_kernel: circular 7x7 convolution of |F|
  * 125-140  spectrum_enhancement: F *= S^alpha only where S^alpha > 0
  * 142-176  patchwise_normalize: S /= mean(S) if mean > 1e-8 else 0
  * 227-274  batched_overlap_add_kernel: triangular weight wx+wy, 1/n^2 scale
  * 280-292  normalize_output_kernel: out /= wsum where wsum > 0
  * 298-323  extract_patches_kernel: patch origin clamped to the image edge
  * 334-341  patch grid: step n/4, ceil(nrow/step) - 3 patches (>= 1)
cuFFT (a closed library; its arithmetic is not restated) is replaced by
float64 ``numpy.fft``; the inverse is unnormalised like cuFFT's.
The reference accumulates into ``d_out`` without clearing it per file
(goldstein.cu:484 clears only the weights); this oracle starts from zero,
which is what the first file of a run sees on a fresh allocation.
"""
from __future__ import annotations

import numpy as np

# goldstein.cu:43-52, row-major (ky, kx) for ky, kx in -3..3.
GAUSS7 = np.array([
    0.000004, 0.000088, 0.000543, 0.000948, 0.000543, 0.000088, 0.000004,
    0.000088, 0.001915, 0.011776, 0.020584, 0.011776, 0.001915, 0.000088,
    0.000543, 0.011776, 0.072410, 0.126584, 0.072410, 0.011776, 0.000543,
    0.000948, 0.020584, 0.126584, 0.221141, 0.126584, 0.020584, 0.000948,
    0.000543, 0.011776, 0.072410, 0.126584, 0.072410, 0.011776, 0.000543,
    0.000088, 0.001915, 0.011776, 0.020584, 0.011776, 0.001915, 0.000088,
    0.000004, 0.000088, 0.000543, 0.000948, 0.000543, 0.000088, 0.000004,
], dtype=np.float32).reshape(7, 7)


def patch_grid(nrow, ncol, n_win):
    """goldstein.cu:334-341 -> (n_inc, n_win_i, n_win_j)."""
    n_inc = n_win // 4
    n_win_i = int(np.ceil(np.float32(nrow) / np.float32(n_inc))) - 3
    n_win_j = int(np.ceil(np.float32(ncol) / np.float32(n_inc))) - 3
    n_win_i = max(n_win_i, 1)
    n_win_j = max(n_win_j, 1)
    return n_inc, n_win_i, n_win_j


def patch_origin(pi, pj, n_win, n_inc, nrow, ncol):
    """goldstein.cu:308-313."""
    i1 = pi * n_inc
    j1 = pj * n_inc
    if i1 + n_win > nrow:
        i1 = nrow - n_win
    if j1 + n_win > ncol:
        j1 = ncol - n_win
    return i1, j1


def tri_weights(n_win):
    """goldstein.cu:257-259 -> [n, n] float32 with w[ty, tx] = wx + wy."""
    t = np.arange(n_win)
    w1 = np.where(t < n_win // 2, t, n_win - 1 - t).astype(np.float32)
    return w1[None, :] + w1[:, None]


def filter_patch(p, alpha):
    """One patch: FFT -> smooth |F| -> normalise -> ^alpha -> IFFT (float64)."""
    n = p.shape[0]
    F = np.fft.fft2(p.astype(np.complex128))
    mag = np.abs(F)
    S = np.zeros_like(mag)
    for ky in range(-3, 4):
        for kx in range(-3, 4):
            # S[y, x] += |F|[(y+ky) mod n, (x+kx) mod n] * G[ky+3, kx+3]
            S += np.roll(mag, shift=(-ky, -kx), axis=(0, 1)) * float(GAUSS7[ky + 3, kx + 3])
    mean = S.sum() / (n * n)
    S = S / mean if mean > 1e-8 else np.zeros_like(S)
    w = np.power(S, alpha)
    F = np.where(w > 0, F * w, F)
    return np.fft.ifft2(F) * (n * n)  # unnormalised inverse, like cuFFT


def goldstein(img, n_win=32, alpha=0.5):
    """goldstein_filter_cuda_host, goldstein.cu:328-408, in float64; returns complex64."""
    nrow, ncol = img.shape
    if nrow < n_win or ncol < n_win:
        raise ValueError("image smaller than the Goldstein window")
    n_inc, n_win_i, n_win_j = patch_grid(nrow, ncol, n_win)
    w = tri_weights(n_win).astype(np.float64)
    norm = 1.0 / (n_win * n_win)
    acc = np.zeros((nrow, ncol), dtype=np.complex128)
    wsum = np.zeros((nrow, ncol), dtype=np.float64)
    for pi in range(n_win_i):
        for pj in range(n_win_j):
            i1, j1 = patch_origin(pi, pj, n_win, n_inc, nrow, ncol)
            f = filter_patch(img[i1:i1 + n_win, j1:j1 + n_win], alpha)
            acc[i1:i1 + n_win, j1:j1 + n_win] += f * w * norm
            wsum[i1:i1 + n_win, j1:j1 + n_win] += w
    out = np.where(wsum > 0, acc / np.where(wsum > 0, wsum, 1.0), acc)
    return out.astype(np.complex64)
