"""The allocation-free gradient entry point, dicegpu_image_gradients_noalloc.

It serves callers that cannot call cudaMalloc themselves (a host that owns all
device memory through its own pool, a per-frame loop that cannot afford
cudaFree's device-wide wait): its scratch planes live in a file-scope device
array instead of a per-call allocation.  Checked through the C ABI against
the allocating entry point, dicegpu_image_gradients, on two calls in a row,
bit for bit (the bar of the other gradient tests).  This file is collected
last so that a stop-at-first-failure run has already run every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

from dice_b200 import abi

pytestmark = pytest.mark.gpu

MAX_PIXELS = 1024 * 1024


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _gradients(fn, img, method):
    h, w = img.shape
    gx = torch.full_like(img, float("nan"))
    gy = torch.full_like(img, float("nan"))
    rc = fn(w, h, _ptr(img), _ptr(gx), _ptr(gy), method, None)
    assert rc == 0, rc
    torch.cuda.synchronize()
    return gx.cpu().numpy(), gy.cpu().numpy()


@pytest.mark.parametrize("method", [abi.CONVOLUTION_5_POINT, abi.FINITE_DIFFERENCE])
def test_noalloc_gradients_match_allocating_entry(method):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = abi.load_library()
    rng = np.random.default_rng(11)
    shapes = [(300, 417), (512, 384)]      # two calls in a row, different sizes and contents
    for h, w in shapes:
        img = torch.from_numpy((rng.random((h, w)) * 65535).astype(np.float32)).cuda()
        ref_gx, ref_gy = _gradients(lib.dicegpu_image_gradients, img, method)
        gx, gy = _gradients(lib.dicegpu_image_gradients_noalloc, img, method)
        assert np.array_equal(gx, ref_gx)
        assert np.array_equal(gy, ref_gy)


def test_noalloc_finite_difference_takes_any_size():
    """The finite-difference method uses no scratch planes, so images larger
    than the 5-point method's cap are computed, equal to the allocating
    entry point's."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = abi.load_library()
    rng = np.random.default_rng(12)
    h, w = 1100, 1031
    assert h * w > MAX_PIXELS
    img = torch.from_numpy((rng.random((h, w)) * 255).astype(np.float32)).cuda()
    ref_gx, ref_gy = _gradients(lib.dicegpu_image_gradients, img, abi.FINITE_DIFFERENCE)
    gx, gy = _gradients(lib.dicegpu_image_gradients_noalloc, img, abi.FINITE_DIFFERENCE)
    assert np.array_equal(gx, ref_gx)
    assert np.array_equal(gy, ref_gy)


def test_noalloc_rejects_images_beyond_its_scratch():
    """The 5-point method's cap: one row over 1024 x 1024 is rejected."""
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = abi.load_library()
    img = torch.zeros((1025, 1024), dtype=torch.float32, device="cuda")
    assert 1025 * 1024 > MAX_PIXELS
    gx = torch.empty_like(img)
    gy = torch.empty_like(img)
    rc = lib.dicegpu_image_gradients_noalloc(1024, 1025, _ptr(img), _ptr(gx), _ptr(gy),
                                             abi.CONVOLUTION_5_POINT, None)
    assert rc == -1
