"""s1b_goldstein_noalloc: the Goldstein filter for callers that cannot
allocate device memory while they filter (a plugin inside an application
whose pool allocator already holds the GPU, or a pipeline that forbids
allocation after start-up).  It uses a fixed device array compiled into the
library instead of caller scratch.

Called through the C ABI (ctypes on libs1b.so) and compared with
s1b_goldstein, the entry point that takes caller scratch, on two calls in a
row (the second with a different image, so stale scratch contents from the
first call would show).  This file is collected last so that a failure here
leaves the rest of the suite already run.
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


def _with_scratch(lib, img, alpha):
    nrow, ncol = img.shape
    need = lib.s1b_goldstein_scratch_bytes(nrow, ncol, 32)
    scratch = torch.empty(need, dtype=torch.uint8, device=img.device)
    out = torch.empty_like(img)
    st = lib.s1b_goldstein(ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()), nrow, ncol, 32,
                           ctypes.c_float(alpha), ctypes.c_void_p(scratch.data_ptr()), need,
                           ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.s1b_last_error()
    return out


def _no_alloc(lib, img, alpha):
    nrow, ncol = img.shape
    out = torch.empty_like(img)
    st = lib.s1b_goldstein_noalloc(ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(out.data_ptr()), nrow, ncol,
                                   32, ctypes.c_float(alpha),
                                   ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 0, lib.s1b_last_error()
    return out


def test_no_alloc_matches_scratch_entry_point_twice(cuda):
    lib = _lib.load()
    for seed, shape, alpha in ((1, (160, 224), 0.5), (2, (96, 130), 0.6)):
        img = _img(seed, *shape)
        want = _with_scratch(lib, img, alpha)
        got = _no_alloc(lib, img, alpha)
        torch.cuda.synchronize()
        g, w = got.cpu().numpy(), want.cpu().numpy()
        assert rel_err(g, w) < 1e-5
        assert phase_rms(g, w) < 1e-3


def test_no_alloc_rejects_images_above_its_limit(cuda):
    lib = _lib.load()
    # 600 x 600 needs 72 x 72 = 5184 patches > S1B_GOLDSTEIN_NOALLOC_MAX_PATCHES
    img = torch.zeros((600, 600), dtype=torch.complex64, device=cuda)
    st = lib.s1b_goldstein_noalloc(ctypes.c_void_p(img.data_ptr()), ctypes.c_void_p(img.data_ptr()), 600, 600, 32,
                                   ctypes.c_float(0.5), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == _lib.S1B_ERR_TOO_LARGE
    assert b"4096" in lib.s1b_last_error()
