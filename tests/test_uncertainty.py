"""Uncertainty fields of Objective::computeUncertaintyFields
(DICe_Objective.cpp:193-299): FIELD_1..FIELD_7, written whenever a subset's
Gauss-Newton solve converges.

CPU: the oracle's restatement against an independent numpy evaluation of the
same formulas (reference-gradient mode, where the subset's gradients are the
reference image's at the pixel), and both against the bitmap_star regression's
gold (its UNCERTAINTY column is SIGMA / FIELD_1).  GPU: parity with the oracle in both gradient
modes through the C ABI.
"""
import ctypes

import numpy as np
import pytest

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O

U = abi.UNCERTAINTY_STRIDE


def _case(w=160, h=128, step=16, **kw):
    ref, deff = syn.config1(w=w, h=h)
    ref, deff = ref.numpy(), deff.numpy()
    cx, cy = syn.grid_points(w, h, 21, step)
    base = dict(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                fast_solver_tolerance=1e-5)
    base.update(kw)
    return ref, deff, cx, cy, abi.default_params(**base)


def _numpy_fields(ref, deff, p, row):
    """The reference's formulas in float64 for one square subset, with the
    reference-image gradients (use_def_gradients = 0)."""
    gxr, gyr = O.gradients(ref)
    cx, cy = int(row[abi.F_COORD_X]), int(row[abi.F_COORD_Y])
    hs = p.subset_size // 2
    ys, xs = np.mgrid[cy - hs:cy + hs + 1, cx - hs:cx + hs + 1]
    xs, ys = xs.ravel(), ys.ravel()
    gx = gxr[ys, xs].astype(np.float64)
    gy = gyr[ys, xs].astype(np.float64)
    u, v = row[abi.F_DISP_X], row[abi.F_DISP_Y]
    g2 = gx * gx + gy * gy
    inv = np.where(g2 < 1e-4, 0.0, 1.0 / np.where(g2 == 0, 1.0, g2))
    a = u * gx + v * gy
    j = v * gx - u * gy
    pts = np.stack([xs + u, ys + v], 1).astype(np.float32)
    at, _, _ = O.interpolate(abi.KEYS_FOURTH, deff, pts)
    at0, _, _ = O.interpolate(abi.KEYS_FOURTH, deff, np.stack([xs, ys], 1).astype(np.float32))
    d = at.astype(np.float64) - at0.astype(np.float64)
    n = len(xs)
    s_uhat = n * (u * u + v * v)
    cos_hat = 1.0 if s_uhat == 0 else np.sqrt((a * a * inv).sum() / s_uhat)
    int_r = (d * d * inv).sum()
    return np.array([cos_hat, 1.0, np.sqrt((a * a * inv).sum() + (j * j * inv).sum()),
                     0.0 if cos_hat == 0 else np.sqrt(int_r) / cos_hat, np.sqrt((a * a * inv).sum()),
                     np.sqrt(int_r), (1.0 + g2.sum()) / n])


def test_oracle_uncertainty_matches_formulas():
    ref, deff, cx, cy, p = _case(use_def_gradients=0)
    f = syn.init_fields(cx, cy)
    unc = np.zeros((len(cx), U))
    O.execute_frame(p, ref, deff, f, first_frame=True, nthreads=4, uncertainty=unc)
    ok = f[:, abi.F_STATUS] < 2
    assert ok.mean() > 0.9
    # every converged Gauss-Newton solve wrote its row
    assert np.all(unc[ok, 1] == 1.0)
    for i in np.nonzero(ok)[0][:12]:
        want = _numpy_fields(ref, deff, p, f[i])
        got = unc[i, :7]
        assert np.allclose(got, want, rtol=2e-4, atol=1e-6), (i, got, want)


# ---- pinned to the reference: bitmap_star --------------------------------------
# The regression's gold prints UNCERTAINTY = SIGMA / FIELD_1 for 2-D results
# (Uncertainty_Post_Processor::execute, DICe_PostProcessor.cpp:1507-1537), so
# FIELD_1 = SIGMA / UNCERTAINTY is a reference vector of computeUncertaintyFields'
# first field.  Fixture: every 20th gold row and 45 x 45 patches of the DIC
# challenge wave pair around those subsets (tests/golden/make_fixtures.py).

def _bitmap_star():
    import os
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_gold.npz"))
    cols = {c: i for i, c in enumerate(str(gold["bitmap_star_columns"]).split(","))}
    rows = gold["bitmap_star_gold"]
    h, w = (int(v) for v in gold["bitmap_star_shape"])
    imgs = []
    for key in ("ref", "def"):
        canvas = np.zeros((h + 44, w + 44), np.float32)
        for (x, y), patch in zip(rows[:, 1:3].astype(int), gold["bitmap_star_%s_patches" % key]):
            canvas[y:y + 45, x:x + 45] = patch
        imgs.append(canvas[22:22 + h, 22:22 + w].copy())
    # file-fed images: the subsets keep the reference image's gradients
    p = abi.default_params(subset_size=31, use_def_gradients=0, compute_uncertainty=1,
                           optimization=abi.GRADIENT_BASED)
    return imgs[0], imgs[1], rows, cols, p


def test_uncertainty_formula_pinned_to_bitmap_star_gold():
    ref, deff, rows, cols, p = _bitmap_star()
    implied = rows[:, cols["SIGMA"]] / rows[:, cols["UNCERTAINTY"]]
    got = []
    for r in rows:
        row = np.zeros(abi.FIELD_STRIDE)
        row[abi.F_COORD_X], row[abi.F_COORD_Y] = r[cols["COORDINATE_X"]], r[cols["COORDINATE_Y"]]
        row[abi.F_DISP_X], row[abi.F_DISP_Y] = r[cols["DISPLACEMENT_X"]], r[cols["DISPLACEMENT_Y"]]
        got.append(_numpy_fields(ref, deff, p, row)[0])
    rel = np.abs(np.array(got) - implied) / implied
    # five printed digits of SIGMA, UNCERTAINTY, u and v (4.8e-5 reached)
    assert rel.max() < 1e-4, rel.max()


def test_oracle_uncertainty_against_bitmap_star_gold():
    ref, deff, rows, cols, p = _bitmap_star()
    f = np.zeros((len(rows), abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = rows[:, cols["COORDINATE_X"]]
    f[:, abi.F_COORD_Y] = rows[:, cols["COORDINATE_Y"]]
    unc = np.zeros((len(rows), U))
    O.execute_frame(p, ref, deff, f, first_frame=True, nthreads=4, uncertainty=unc)
    assert np.all(f[:, abi.F_STATUS] < 2)
    # the reference started each solve from feature matching, these from zero:
    # the solves stop within the 1e-4 px tolerance of each other
    assert np.abs(f[:, abi.F_DISP_X] - rows[:, cols["DISPLACEMENT_X"]]).max() < 1e-4
    assert np.abs(f[:, abi.F_DISP_Y] - rows[:, cols["DISPLACEMENT_Y"]]).max() < 1e-4
    # where u and v stop apart, FIELD_1 moves with their direction
    rel = np.abs(f[:, abi.F_SIGMA] / unc[:, 0] - rows[:, cols["UNCERTAINTY"]]) / rows[:, cols["UNCERTAINTY"]]
    assert (rel < 1e-4).mean() > 0.95 and rel.max() < 1e-2, (np.median(rel), rel.max())
    _check_sigma_gamma(f, rows, cols)


def _check_sigma_gamma(f, rows, cols):
    for name, c in (("SIGMA", abi.F_SIGMA), ("GAMMA", abi.F_GAMMA)):
        rel = np.abs(f[:, c] - rows[:, cols[name]]) / rows[:, cols[name]]
        assert (rel < 1e-4).mean() > 0.95 and rel.max() < 1e-2, (name, rel.max())


def test_oracle_uncertainty_untouched_without_convergence():
    ref, deff, cx, cy, p = _case(use_def_gradients=0, optimization=abi.SIMPLEX)
    f = syn.init_fields(cx, cy)
    unc = np.zeros((len(cx), U))
    O.execute_frame(p, ref, deff, f, first_frame=True, nthreads=4, uncertainty=unc)
    assert not unc.any()          # the simplex never writes them


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
@pytest.mark.parametrize("defgrad", [0, 1])
def test_gpu_uncertainty_matches_oracle(defgrad):
    _gpu()
    from dice_b200.schema import Schema
    ref, deff, cx, cy, p = _case(w=256, h=192, step=12, use_def_gradients=defgrad, compute_uncertainty=1)
    f = syn.init_fields(cx, cy)
    # two frames: the rows persist and are rewritten by the second solve
    frames = [deff, syn.warp_image(syn.config1(w=256, h=192)[0], lambda X, Y: (0.6 + 0 * X, -1.0 + 0 * Y),
                                   noise_sigma=2.0, seed=9, clip=(0, 255)).numpy()]
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        got = []
        for d in frames:
            s.set_def_image(d)
            s.execute_correlation()
            got.append((s.fields(), s.uncertainty()))
    o = f.copy()
    unc = np.zeros((len(cx), U))
    for k, d in enumerate(frames):
        O.execute_frame(p, ref, d, o, first_frame=(k == 0), nthreads=4, uncertainty=unc)
        g, gu = got[k]
        assert np.array_equal(g[:, abi.F_STATUS], o[:, abi.F_STATUS])
        ok = (o[:, abi.F_STATUS] < 2) & (g[:, abi.F_ITERATIONS] == o[:, abi.F_ITERATIONS])
        assert ok.mean() > 0.9
        # u, v agree to 1e-4 px between the two, which bounds the fields'
        # agreement (FIELD_4/6 scale with the displacement)
        assert np.allclose(gu[ok, :7], unc[ok, :7], rtol=2e-3, atol=1e-5)
        assert np.all(gu[ok, 1] == 1.0)


@pytest.mark.gpu
def test_gpu_uncertainty_against_bitmap_star_gold():
    _gpu()
    from dice_b200.schema import Schema
    ref, deff, rows, cols, p = _bitmap_star()
    f = np.zeros((len(rows), abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = rows[:, cols["COORDINATE_X"]]
    f[:, abi.F_COORD_Y] = rows[:, cols["COORDINATE_Y"]]
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        s.set_def_image(deff)
        s.execute_correlation()
        g, gu = s.fields(), s.uncertainty()
    assert np.all(g[:, abi.F_STATUS] < 2)
    rel = np.abs(g[:, abi.F_SIGMA] / gu[:, 0] - rows[:, cols["UNCERTAINTY"]]) / rows[:, cols["UNCERTAINTY"]]
    assert (rel < 1e-4).mean() > 0.95 and rel.max() < 1e-2, (np.median(rel), rel.max())
    _check_sigma_gamma(g, rows, cols)


@pytest.mark.gpu
def test_gpu_uncertainty_requires_the_option():
    _gpu()
    from dice_b200.schema import Schema
    ref, deff, cx, cy, p = _case()
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_subsets(cx, cy)
        s.set_def_image(deff)
        s.execute_correlation()
        out = np.zeros((len(cx), U))
        rc = s.lib.dicegpu_get_uncertainty(s.ctx, out.ctypes.data_as(ctypes.c_void_p))
        assert rc == abi.ERR_STATE
