"""GPU parity: libdicegpu.so (through its C ABI) against the CPU oracle.

The bar is equality: the library computes the reference's float operations
in the reference's order (interpolation weights in double, 2-D tap sums,
sequential float means and gamma / sigma / noise sums, float-rounded products
in the double Hessian and right-hand side, LU factors and explicit inverse,
the update accumulated in float), so every result column -- status,
iterations, parameters, sigma, gamma, noise, contrast, active pixels,
condition number -- equals the oracle's bit for bit.  The double sums run in
another order than the reference's sequential one; that moves them by about
1e-16 relative, which decides a float rounding of the parameter update only
with a probability of order 1e-9 per update, so none occurs in these cases.
"""
import numpy as np
import pytest
import torch

from dice_b200 import abi
from dice_b200.schema import Schema, correlate
from dice_b200 import synthetic as syn
from oracle import oracle as O
from tests._exact import assert_rows_equal

pytestmark = pytest.mark.gpu

def _require_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _run_gpu(params, ref, deff, fields, frames=None, lists=None, force=None, plain=False):
    s = Schema(params)
    s.set_ref_image(ref)
    s.set_fields(fields)
    if lists is not None:
        s.set_subset_pixels(*lists)
    if force is not None:
        s.set_force_simplex(force)
    out = []
    for d in (frames if frames is not None else [deff]):
        s.set_def_image(d)
        if plain:
            s.execute_correlation_plain()
        else:
            s.execute_correlation()
        out.append(s.fields())
    assert s.device_status() == 0
    s.close()
    return out


def _run_oracle(params, ref, deff, fields, frames=None, lists=None, force=None):
    f = fields.copy()
    out = []
    for k, d in enumerate(frames if frames is not None else [deff]):
        kw = {}
        if lists is not None:
            kw = dict(offsets=lists[0], px=lists[1], py=lists[2])
        O.execute_frame(params, np.asarray(ref), np.asarray(d), f, first_frame=(k == 0), nthreads=8,
                        force_simplex=force, **kw)
        out.append(f.copy())
    return out


def _compare(g, o):
    assert_rows_equal(g, o)


def test_gradients_bit_exact():
    _require_gpu()
    lib = abi.load_library()
    rng = np.random.default_rng(7)
    img = (rng.random((97, 131)) * 65535).astype(np.float32)
    for method in (abi.FINITE_DIFFERENCE, abi.CONVOLUTION_5_POINT):
        gx_o, gy_o = O.gradients(img, method)
        t = torch.from_numpy(img).cuda()
        gx = torch.empty_like(t)
        gy = torch.empty_like(t)
        import ctypes
        rc = lib.dicegpu_image_gradients(131, 97, ctypes.c_void_p(t.data_ptr()), ctypes.c_void_p(gx.data_ptr()),
                                         ctypes.c_void_p(gy.data_ptr()), method, None)
        assert rc == 0
        torch.cuda.synchronize()
        assert np.array_equal(gx.cpu().numpy(), gx_o)
        assert np.array_equal(gy.cpu().numpy(), gy_o)


@pytest.mark.parametrize("method", [abi.KEYS_FOURTH, abi.BICUBIC, abi.BILINEAR])
def test_interpolate_matches_oracle(method):
    _require_gpu()
    ref, deff = syn.config1(w=128, h=96)
    ref, deff = ref.numpy(), deff.numpy()
    rng = np.random.default_rng(3)
    # the whole image and a margin around it: border fallbacks and the
    # kernel sums that overwrite them, taps outside the image read as 0
    xy = np.stack([rng.uniform(-1.5, 127.4, 20000), rng.uniform(-1.5, 95.4, 20000)], 1).astype(np.float32)
    with Schema(abi.default_params()) as s:
        s.set_ref_image(ref)
        s.set_def_image(deff)
        gi, ggx, ggy = s.interpolate(method, xy)
    dgx, dgy = O.gradients(deff)
    oi, ogx, ogy = O.interpolate(method, deff, xy, dgx, dgy)
    assert np.array_equal(gi, oi)
    assert np.array_equal(ggx, ogx)
    assert np.array_equal(ggy, ogy)


def test_reference_gold_on_gpu(gold):
    """parallel_subsets gold (file-fed images: reference-gradient mode)."""
    _require_gpu()
    ref = gold["ref_speckled"].astype(np.float32)
    de = gold["def_speckled"].astype(np.float32)
    g = gold["parallel_subsets_gold"]
    p = abi.default_params(subset_size=27, use_def_gradients=0)
    f = syn.init_fields(g[:, 1], g[:, 2])
    gpu = _run_gpu(p, ref, de, f)[0]
    ora = _run_oracle(p, ref, de, f)[0]
    _compare(gpu, ora)
    assert np.all(gpu[:, abi.F_ITERATIONS] == g[:, 9])
    assert np.all(gpu[:, abi.F_STATUS] == g[:, 10])
    assert np.max(np.abs(gpu[:, abi.F_DISP_X] - g[:, 3])) < 1e-4
    assert np.max(np.abs(gpu[:, abi.F_DISP_Y] - g[:, 4])) < 1e-4


def test_single_speckled_shift_sigma_on_gpu(gold):
    _require_gpu()
    ref = gold["ref_speckled"].astype(np.float32)
    de = gold["def_speckled"].astype(np.float32)
    s = gold["single_speckled_shift_gold"]
    p = abi.default_params(subset_size=27, use_def_gradients=0)
    gpu = _run_gpu(p, ref, de, syn.init_fields(s[:, 1], s[:, 2]))[0]
    assert np.all(gpu[:, abi.F_STATUS] == s[:, 10])
    assert np.max(np.abs(gpu[:, abi.F_SIGMA] - s[:, 9]) / s[:, 9]) < 2e-4
    assert np.max(np.abs(gpu[:, abi.F_DISP_X] - s[:, 3])) < 1e-4


def _config1_params(**kw):
    base = dict(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                fast_solver_tolerance=1e-5, max_solver_iterations_fast=25)
    base.update(kw)
    return abi.default_params(**base)


def test_config1_affine_parity():
    """512^2, 21x21 subsets at step 10 (2304), affine 6 parameters, tol 1e-5."""
    _require_gpu()
    ref, deff = syn.config1()
    cx, cy = syn.grid_points(512, 512, 21, 10)
    assert len(cx) == 2304
    p = _config1_params()
    f = syn.init_fields(cx, cy)
    gpu = _run_gpu(p, ref.numpy(), deff.numpy(), f)[0]
    ora = _run_oracle(p, ref.numpy(), deff.numpy(), f)[0]
    _compare(gpu, ora)
    ok = ora[:, abi.F_STATUS] < 2
    assert ok.mean() > 0.99
    # imposed field: u = 0.37, v = -1.21
    assert np.abs(np.median(gpu[ok, abi.F_DISP_X]) - 0.37) < 0.01
    assert np.abs(np.median(gpu[ok, abi.F_DISP_Y]) + 1.21) < 0.01


@pytest.mark.parametrize("interp", [abi.BICUBIC, abi.BILINEAR])
def test_other_interpolants_parity(interp):
    _require_gpu()
    ref, deff = syn.config1(w=256, h=256)
    cx, cy = syn.grid_points(256, 256, 21, 12)
    p = _config1_params(interpolation=interp)
    f = syn.init_fields(cx, cy)
    gpu = _run_gpu(p, ref.numpy(), deff.numpy(), f)[0]
    ora = _run_oracle(p, ref.numpy(), deff.numpy(), f)[0]
    _compare(gpu, ora)


def test_multiframe_sequence_parity():
    """Frames initialised from the previous solution (config 2 field, reduced size)."""
    _require_gpu()
    w = h = 384
    ref = syn.speckle_image(w, h, seed=2, r_min=3, r_max=5, grey_lo=1000, grey_hi=64000, blur_sigma=0.8)
    frames = [syn.warp_image(ref, syn.config2_field(k + 1, 4), noise_sigma=50.0, seed=200 + k,
                             clip=(0, 65535)).numpy() for k in range(4)]
    cx, cy = syn.grid_points(w, h, 31, 9)
    p = _config1_params(subset_size=31)
    f = syn.init_fields(cx, cy)
    gpu = _run_gpu(p, ref.numpy(), None, f, frames=frames)
    ora = _run_oracle(p, ref.numpy(), None, f, frames=frames)
    for g, o in zip(gpu, ora):
        _compare(g, o)


def test_plain_path_matches_batched():
    _require_gpu()
    ref, deff = syn.config1(w=256, h=256)
    cx, cy = syn.grid_points(256, 256, 21, 15)
    p = _config1_params()
    f = syn.init_fields(cx, cy)
    a = _run_gpu(p, ref.numpy(), deff.numpy(), f)[0]
    b = _run_gpu(p, ref.numpy(), deff.numpy(), f, plain=True)[0]
    assert np.array_equal(a, b)


def test_simplex_parity():
    _require_gpu()
    ref, deff = syn.config1(w=192, h=192)
    cx, cy = syn.grid_points(192, 192, 21, 20)
    p = abi.default_params(subset_size=21, optimization=abi.SIMPLEX, enable_rotation=1)
    f = syn.init_fields(cx, cy)
    gpu = _run_gpu(p, ref.numpy(), deff.numpy(), f)[0]
    ora = _run_oracle(p, ref.numpy(), deff.numpy(), f)[0]
    _compare(gpu, ora)
    ok = ora[:, abi.F_STATUS] < 2
    assert np.abs(np.median(gpu[ok, abi.F_DISP_X]) - 0.37) < 0.02


def test_quadratic_parity():
    _require_gpu()
    ref, deff = syn.config1(w=256, h=256)
    cx, cy = syn.grid_points(256, 256, 31, 20)
    p = abi.default_params(subset_size=31, shape_function=abi.QUADRATIC_SF, fast_solver_tolerance=1e-5)
    f = syn.init_fields(cx, cy, quadratic=True)
    gpu = _run_gpu(p, ref.numpy(), deff.numpy(), f)[0]
    ora = _run_oracle(p, ref.numpy(), deff.numpy(), f)[0]
    _compare(gpu, ora)


def test_pixel_list_subsets_parity():
    """Arbitrary-shape subsets (circles) given as pixel lists."""
    _require_gpu()
    ref, deff = syn.config1(w=256, h=256)
    rng = np.random.default_rng(5)
    cx = rng.integers(40, 216, 60)
    cy = rng.integers(40, 216, 60)
    offs, px, py = [0], [], []
    for x0, y0 in zip(cx, cy):
        r = rng.integers(7, 16)
        for yy in range(y0 - r, y0 + r + 1):
            for xx in range(x0 - r, x0 + r + 1):
                if (xx - x0) ** 2 + (yy - y0) ** 2 <= r * r:
                    px.append(xx)
                    py.append(yy)
        offs.append(len(px))
    lists = (np.asarray(offs), np.asarray(px), np.asarray(py))
    p = _config1_params(subset_size=0)
    f = syn.init_fields(cx.astype(float), cy.astype(float))
    gpu = _run_gpu(p, ref.numpy(), deff.numpy(), f, lists=lists)[0]
    ora = _run_oracle(p, ref.numpy(), deff.numpy(), f, lists=lists)[0]
    _compare(gpu, ora)


def test_failure_flags_match():
    """Host-made failures: flat regions, subsets leaving the image, a failed
    frame's INITIALIZE_FAILED on the next frame (DICe_Initializer.cpp:415-435)."""
    _require_gpu()
    w = h = 160
    ref, deff = syn.config1(w=w, h=h)
    ref = ref.numpy().copy()
    deff = deff.numpy().copy()
    ref[:, :60] = 100.0            # flat: zero gradients / zero contrast
    deff[:, :60] = 100.0
    cx = np.array([30, 100, 120, 150, 5, 80], float)
    cy = np.array([80, 80, 40, 80, 80, 150], float)
    p = abi.default_params(subset_size=21)
    f = syn.init_fields(cx, cy)
    f[3, abi.F_DISP_X] = 30.0      # pushes the subset out of the image
    gpu = _run_gpu(p, ref, None, f, frames=[deff, deff])
    ora = _run_oracle(p, ref, None, f, frames=[deff, deff])
    for g, o in zip(gpu, ora):
        assert np.array_equal(g[:, abi.F_STATUS], o[:, abi.F_STATUS]), (g[:, abi.F_STATUS], o[:, abi.F_STATUS])
        assert np.array_equal(g[:, abi.F_SIGMA] == -1, o[:, abi.F_SIGMA] == -1)


def _api_oracle_frame(p, ref, de, rows, pts, first):
    """One dice_correlate call on the oracle: the nine stride-9 columns
    written over the kept rows, one frame, the results read back as floats."""
    cols = [abi.F_COORD_X, abi.F_COORD_Y, abi.F_DISP_X, abi.F_DISP_Y, abi.F_ROT_Z, abi.F_SIGMA, abi.F_GAMMA,
            abi.F_BETA, abi.F_STATUS]
    rows[:, cols] = pts.astype(np.float64)
    O.execute_frame(p, ref, de, rows, first_frame=first, nthreads=4)
    out = pts.copy()
    out[:, 2:] = rows[:, cols[2:]].astype(np.float32)
    return out


def test_correlate_stride9_api(gold):
    """DICe_TestAPI: integer shifts 0..5 of a 100x100 synthetic speckle image
    through the stride-9 dice_correlate interface (tracking defaults), six
    calls on the one context the library keeps (the reference's static
    Schema): every call's results equal the oracle run as a six-frame
    sequence, and the shifts are recovered."""
    _require_gpu()
    from dice_b200.schema import correlate_reset
    correlate_reset()
    ref = gold["def_synthetic_0"].astype(np.float32)
    pts = np.zeros((4, 9), np.float32)
    pts[:, 0] = [47, 51, 51, 47]
    pts[:, 1] = [47, 47, 51, 51]
    p = abi.tracking_default_params(subset_size=21, use_def_gradients=1)
    rows = np.zeros((4, abi.FIELD_STRIDE))
    want = pts.copy()
    try:
        for k in range(6):
            de = gold["def_synthetic_%d" % k].astype(np.float32)
            want = _api_oracle_frame(p, ref, de, rows, want, k == 0)
            assert correlate(pts, 21, ref, de) == 0
            assert np.array_equal(pts, want), (k, pts, want)
            assert np.all(np.abs(pts[:, 2] - k) < 1e-4), pts
            assert np.all(np.abs(pts[:, 3] - k) < 1e-4), pts
            assert np.all(np.abs(pts[:, 4]) < 1e-4)
            assert np.all(pts[:, 6] < 1e-4)
            assert np.all(pts[:, 8] == 1)
    finally:
        correlate_reset()


def test_correlate_keeps_its_context_until_reset(gold):
    """What the kept context fixes: later calls ignore the reference image and
    the subset size, reject another subset count, and read new parameters
    only with update_params; after dicegpu_correlate_reset the next call
    starts a new sequence."""
    _require_gpu()
    from dice_b200.schema import correlate_reset
    correlate_reset()
    ref = gold["def_synthetic_0"].astype(np.float32)
    d1 = gold["def_synthetic_1"].astype(np.float32)
    d2 = gold["def_synthetic_2"].astype(np.float32)
    start = np.zeros((4, 9), np.float32)
    start[:, 0] = [47, 51, 51, 47]
    start[:, 1] = [47, 47, 51, 51]
    p = abi.tracking_default_params(subset_size=21, use_def_gradients=1)
    try:
        pts = start.copy()
        assert correlate(pts, 21, ref, d1) == 0
        # another reference image and subset size are not read again
        rows = np.zeros((4, abi.FIELD_STRIDE))
        want = _api_oracle_frame(p, ref, d1, rows, start.copy(), True)
        want = _api_oracle_frame(p, ref, d2, rows, want, False)
        assert correlate(pts, 41, d1, d2) == 0
        assert np.array_equal(pts, want)
        # another number of subsets is rejected and leaves the context alone
        assert correlate(pts[:3].copy(), 21, ref, d2) == abi.ERR_ARG
        # parameters change only with update_params: without rotation theta
        # stays at its guess
        p_norot = abi.tracking_default_params(enable_rotation=0)
        guess = pts.copy()
        guess[:, 4] = 0.01
        q = guess.copy()
        assert correlate(q, 21, ref, d2, params=p_norot) == 0
        assert np.all(q[:, 4] != np.float32(0.01))
        q = guess.copy()
        assert correlate(q, 21, ref, d2, params=p_norot, update_params=True) == 0
        assert np.all(q[:, 4] == np.float32(0.01))
        # a reset starts a new sequence at the first frame, as a fresh process
        correlate_reset()
        pts = start.copy()
        assert correlate(pts, 21, ref, d1) == 0
        want = _api_oracle_frame(p, ref, d1, np.zeros((4, abi.FIELD_STRIDE)), start.copy(), True)
        assert np.array_equal(pts, want)
    finally:
        correlate_reset()


def test_gamma_entry_matches_oracle():
    _require_gpu()
    ref, deff = syn.config1(w=200, h=200)
    cx, cy = syn.grid_points(200, 200, 21, 25)
    p = _config1_params()
    f = syn.init_fields(cx, cy)
    f[:, abi.F_DISP_X] = 0.37
    f[:, abi.F_DISP_Y] = -1.21
    with Schema(p) as s:
        s.set_ref_image(ref.numpy())
        s.set_def_image(deff.numpy())
        s.set_fields(f)
        g = s.gamma(f)
    o = O.gamma(p, ref.numpy(), deff.numpy(), f)
    assert np.array_equal(g, o)


def test_headline_strip_x_ge_1024_exact():
    """The 2048^2 sequence (31 x 31 affine subsets at step 5, tolerance 1e-5)
    on the strip x in [1024, 2048), y in [900, 1156): there the float spacing
    of mapped coordinates (1.2e-4 px) exceeds the tolerance, the last
    Gauss-Newton updates oscillate at that spacing and rounding decides
    iteration counts and simplex fallbacks.  Four frames, each from the
    previous solution; every result column equal to the oracle's."""
    _require_gpu()
    ref, frames = syn.config2(device="cuda", nframes=10, count=4)
    cx, cy = syn.grid_points(2048, 2048, 31, 5)
    sel = np.nonzero((cx >= 1024) & (cy >= 900) & (cy < 1156))[0]
    assert len(sel) > 10000
    p = _config1_params(subset_size=31)
    f = syn.init_fields(cx[sel], cy[sel])
    ref_h = ref.cpu().numpy()
    frames_h = [fr.cpu().numpy() for fr in frames]
    gpu = _run_gpu(p, ref, None, f, frames=frames)
    ora = _run_oracle(p, ref_h, None, f, frames=frames_h)
    for g, o in zip(gpu, ora):
        _compare(g, o)
    assert (ora[-1][:, abi.F_STATUS] < 2).all()
