"""s1b_goldstein_noalloc: the Goldstein filter for callers that cannot
allocate device memory while they filter (a plugin inside an application
whose pool allocator already holds the GPU, or a pipeline that forbids
allocation after start-up).  It uses a fixed device array compiled into the
library instead of caller scratch.

Called through the C ABI (ctypes on libs1b.so) and compared with
s1b_goldstein, the entry point that takes caller scratch, on calls in a row:
two images of different shapes, two images of the same shape with different
seeds (every patch slot the second call reads is one the first call wrote,
so a slot the second call failed to rewrite would show the first image's
values), an image of exactly S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES patches, and
one filtered in place (in == out).  Sizes one patch row above the limit are
rejected.  This file is collected last so that a failure here leaves the
rest of the suite already run.
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import phase_rms, rel_err
from sentinel_gpu_processor_b200 import _lib

pytestmark = pytest.mark.gpu


def _img(seed, nrow, ncol):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:nrow, 0:ncol]
    z = np.exp(1j * (0.07 * x + 0.05 * y)) + 0.7 * (rng.standard_normal((nrow, ncol)) +
                                                    1j * rng.standard_normal((nrow, ncol)))
    return torch.from_numpy(z.astype(np.complex64)).cuda()


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _with_scratch(lib, img, alpha):
    nrow, ncol = img.shape
    need = lib.s1b_goldstein_scratch_bytes(nrow, ncol, 32)
    scratch = torch.empty(need, dtype=torch.uint8, device=img.device)
    out = torch.empty_like(img)
    st = lib.s1b_goldstein(ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()), nrow, ncol, 32,
                           ctypes.c_float(alpha), ctypes.c_void_p(scratch.data_ptr()), need, _stream())
    assert st == 0, lib.s1b_last_error()
    return out


def _no_alloc(lib, img, alpha, out=None):
    nrow, ncol = img.shape
    out = torch.empty_like(img) if out is None else out
    st = lib.s1b_goldstein_noalloc(ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()), nrow, ncol,
                                   32, ctypes.c_float(alpha), _stream())
    assert st == 0, lib.s1b_last_error()
    return out


def _patches(nrow, ncol):
    return (-(-nrow // 8) - 3) * (-(-ncol // 8) - 3)


def _check(got, want):
    torch.cuda.synchronize()
    g, w = got.cpu().numpy(), want.cpu().numpy()
    assert rel_err(g, w) < 1e-5
    assert phase_rms(g, w) < 1e-3


def test_no_alloc_matches_scratch_entry_point_twice(cuda):
    lib = _lib.load()
    cases = ((1, (160, 224), 0.5), (2, (96, 130), 0.6),   # two shapes
             (3, (200, 264), 0.5), (4, (200, 264), 0.5))  # one shape, two seeds
    for seed, shape, alpha in cases:
        img = _img(seed, *shape)
        _check(_no_alloc(lib, img, alpha), _with_scratch(lib, img, alpha))


def test_no_alloc_at_its_limit_and_in_place(cuda):
    lib = _lib.load()
    assert _patches(536, 536) == _lib.S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES
    img = _img(5, 536, 536)
    want = _with_scratch(lib, img, 0.5)
    _check(_no_alloc(lib, img, 0.5), want)
    inplace = img.clone()
    _check(_no_alloc(lib, inplace, 0.5, out=inplace), want)


def test_no_alloc_rejects_images_above_its_limit(cuda):
    lib = _lib.load()
    for nrow, ncol in ((544, 536), (600, 600)):
        assert _patches(nrow, ncol) > _lib.S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES
        img = torch.zeros((nrow, ncol), dtype=torch.complex64, device=cuda)
        st = lib.s1b_goldstein_noalloc(ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(img.data_ptr()), nrow, ncol,
                                       32, ctypes.c_float(0.5), _stream())
        assert st == _lib.S1B_ERR_TOO_LARGE
        assert b"4096" in lib.s1b_last_error()
