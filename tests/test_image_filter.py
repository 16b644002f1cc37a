"""Gaussian image pre-filter (Image_::gauss_filter, DICe_Image.cpp:1194-1230).

The oracle is pinned to the reference's own filtered images
(DICe_TestImage.cpp:318-410: ImageB.tif through masks 5..13 against
outFilter<M>.rawi).  Those files were written by a build whose float
evaluation order is not the plain loop of the source: the restatement of that
loop matches them to within 3 ulp of full scale (|d| <= 4.6e-5 on values up to 255), far
inside the reference test's own bar (L2 difference < 0.1 over the image).
The GPU kernel is bit-exact with the oracle.
"""
import ctypes
import os

import numpy as np
import pytest

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O
from tests._exact import assert_rows_equal

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_gold.npz"))
MASKS = (5, 7, 9, 11, 13)


@pytest.mark.parametrize("m", MASKS)
def test_oracle_gauss_filter_matches_reference_images(m):
    img = GOLD["image_b"].astype(np.float32)
    y0, x0 = GOLD["gauss_gold_origin"]
    gold = GOLD["gauss_gold_%d" % m]
    out = O.gauss_filter(img, m)[y0:y0 + 64, x0:x0 + 64]
    d = out.astype(np.float64) - gold
    assert np.sqrt((d * d).sum()) < 0.1          # the reference test's bar
    # rounding follows the partial sums, so the bound is 3 ulp of full scale
    assert np.max(np.abs(d)) <= 3 * float(np.spacing(np.float32(255.0)))
    assert (d == 0).mean() > 0.5


def test_oracle_gauss_filter_keeps_border_and_rejects_bad_masks():
    rng = np.random.default_rng(4)
    img = (rng.random((40, 50)) * 255).astype(np.float32)
    out = O.gauss_filter(img, 7)
    half = 7 // 2 + 1
    assert np.array_equal(out[:half], img[:half])
    assert np.array_equal(out[:, -half:], img[:, -half:])
    assert not np.array_equal(out[half:-half, half:-half], img[half:-half, half:-half])
    lib = O.lib()
    for bad in (3, 6, 15):
        assert lib.oracle_gauss_filter(50, 40, img.ctypes.data, out.ctypes.data, bad) != 0


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.gpu
@pytest.mark.parametrize("m", MASKS)
def test_gpu_gauss_filter_bit_exact(m):
    torch = _gpu()
    lib = abi.load_library()
    rng = np.random.default_rng(m)
    for img in (GOLD["image_b"].astype(np.float32), (rng.random((203, 317)) * 65535).astype(np.float32)):
        h, w = img.shape
        t = torch.from_numpy(img).cuda()
        out = torch.empty_like(t)
        rc = lib.dicegpu_gauss_filter(w, h, ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                      m, None)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), O.gauss_filter(img, m))


@pytest.mark.gpu
def test_gpu_gauss_filter_rejects_bad_arguments():
    torch = _gpu()
    lib = abi.load_library()
    t = torch.zeros((8, 8), device="cuda")
    u = torch.zeros((8, 8), device="cuda")
    p, q = ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(u.data_ptr())
    assert lib.dicegpu_gauss_filter(8, 8, p, q, 9, None) == abi.ERR_ARG      # image smaller than the mask
    assert lib.dicegpu_gauss_filter(8, 8, p, q, 4, None) == abi.ERR_ARG      # not a mask size
    assert lib.dicegpu_gauss_filter(8, 8, p, p, 5, None) == abi.ERR_ARG      # in place


@pytest.mark.gpu
@pytest.mark.parametrize("m", [5, 9])
def test_correlation_with_filtered_images_matches_oracle(m):
    _gpu()
    from dice_b200.schema import Schema
    ref, deff = syn.config1(w=192, h=160)
    ref, deff = ref.numpy(), deff.numpy()
    cx, cy = syn.grid_points(192, 160, 21, 12)
    p = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           fast_solver_tolerance=1e-5, gauss_filter_images=1, gauss_filter_mask_size=m)
    f = syn.init_fields(cx, cy)
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        s.set_def_image(deff)
        s.execute_correlation()
        g = s.fields()
    o = f.copy()
    O.execute_frame(p, ref, deff, o, first_frame=True, nthreads=4)
    assert_rows_equal(g, o)
    ok = o[:, abi.F_STATUS] < 2
    assert ok.mean() > 0.9
    # filtering changes the result (the option is not silently ignored)
    p0 = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                            fast_solver_tolerance=1e-5)
    o0 = f.copy()
    O.execute_frame(p0, ref, deff, o0, first_frame=True, nthreads=4)
    assert not np.array_equal(o0[ok, abi.F_GAMMA], o[ok, abi.F_GAMMA])


@pytest.mark.gpu
def test_invalid_filter_mask_rejected_by_params():
    _gpu()
    from dice_b200.schema import Schema
    with pytest.raises(Exception):
        Schema(abi.default_params(gauss_filter_images=1, gauss_filter_mask_size=8))


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", [np.uint8, np.uint16])
@pytest.mark.parametrize("gauss", [0, 1])
def test_integer_images_equal_their_float_values(dtype, gauss):
    """8- and 16-bit frames uploaded as integers correlate exactly like the
    same values uploaded as floats (host and device sources)."""
    torch = _gpu()
    from dice_b200.schema import Schema
    scale = 1.0 if dtype == np.uint8 else 250.0
    ref, deff = syn.config1(w=160, h=128)
    ref_i = np.clip(np.round(ref.numpy() * scale), 0, np.iinfo(dtype).max).astype(dtype)
    def_i = np.clip(np.round(deff.numpy() * scale), 0, np.iinfo(dtype).max).astype(dtype)
    cx, cy = syn.grid_points(160, 128, 21, 12)
    p = abi.default_params(subset_size=21, enable_rotation=1, fast_solver_tolerance=1e-5,
                           gauss_filter_images=gauss, gauss_filter_mask_size=7)
    out = []
    for r, d in ((ref_i.astype(np.float32), def_i.astype(np.float32)), (ref_i, def_i),
                 (torch.from_numpy(ref_i.astype(np.int32)).to(torch.uint16 if dtype == np.uint16 else torch.uint8).cuda(),
                  torch.from_numpy(def_i.astype(np.int32)).to(torch.uint16 if dtype == np.uint16 else torch.uint8).cuda())):
        with Schema(p) as s:
            s.set_ref_image(r)
            s.set_subsets(cx, cy)
            s.set_def_image(d)
            s.execute_correlation()
            out.append(s.fields())
    assert np.array_equal(out[0], out[1])
    assert np.array_equal(out[0], out[2])
    assert np.mean(out[0][:, abi.F_STATUS] < 2) > 0.9
