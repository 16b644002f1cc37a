"""Regular grids of correlation points and VSG strain.

* create_regular_grid_of_correlation_points (DICe_Decomp.cpp:868-1050):
  the dic_challenge_12 region of interest (a 313 x 977 rectangle minus a
  radius-51 circle, step 35, subset 27, 400 x 1040 image) gives exactly the
  reference's 230 points in its snaking order (the unsorted gold) and, sorted,
  the sorted gold's order.
* VSG_Strain_Post_Processor (DICe_PostProcessor.cpp:877-1130): the oracle,
  fed the gold's printed displacements, reproduces the gold's VSG strains
  within the rounding of those five-digit inputs; exact on affine fields;
  the failure cases give zeros and MATCH = -1.  The GPU equals the oracle to
  float rounding and, written through the result writer, passes the
  reference's regression comparison of the dic_challenge_12 files.
"""
import os

import numpy as np
import pytest

from dice_b200 import abi
from dice_b200.results import Output, diff_text
from dice_b200.subset_file import SubsetFile, regular_grid
from oracle import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_gold.npz"))
FRAMES = ("01", "06", "11")
WINDOW = 360


def _rows(text):
    out = []
    for line in text.splitlines():
        line = line.strip()
        if not line or line.startswith("***") or line[0].isalpha():
            continue
        out.append([float(t) for t in line.split(",")])
    return np.asarray(out)


def _gold(variant, k):
    """columns: x, y, u, v, vsg_xx, vsg_yy, gamma, match"""
    return _rows(str(GOLD["%s_gold_text_%s" % (variant, k)]))


def _fields(g):
    f = np.zeros((len(g), abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X], f[:, abi.F_COORD_Y] = g[:, 0], g[:, 1]
    f[:, abi.F_DISP_X], f[:, abi.F_DISP_Y] = g[:, 2], g[:, 3]
    f[:, abi.F_GAMMA], f[:, abi.F_MATCH] = g[:, 6], g[:, 7]
    return f


def test_region_of_interest_grid_matches_reference_order():
    sf = SubsetFile(text=str(GOLD["subset_file_dic_challenge_12"]))
    assert sf.info.region_of_interest == 1
    xy, neigh, seed = regular_grid(sf, 400, 1040, 35, 27)
    for k in FRAMES:
        assert np.array_equal(xy, _gold("dic_challenge_12", k)[:, :2])
    order = np.lexsort((xy[:, 1], xy[:, 0]))
    assert np.array_equal(xy[order], _gold("dic_challenge_12_sorted", "01")[:, :2])
    # the first grid point (26, 26) lies outside the region: no seed, so every
    # point's neighbour is the previous point of its snake
    assert neigh[0] == -1 and np.array_equal(neigh[1:], np.arange(len(xy) - 1)) and (seed == -1).all()


def test_whole_image_grid_and_seeded_region():
    xy, neigh, _ = regular_grid(None, 100, 80, 10, 11)
    xs, ys = np.unique(xy[:, 0]), np.unique(xy[:, 1])
    # from subset_size - 1 in steps, keeping subset_size - 1 from the far edges
    assert xs.tolist() == list(range(10, 90, 10)) and ys.tolist() == list(range(10, 70, 10))
    assert len(xy) == len(xs) * len(ys)
    text = ("BEGIN REGION_OF_INTEREST\nBEGIN BOUNDARY\nBEGIN RECTANGLE\nCENTER 50 40\nWIDTH 100\nHEIGHT 80\nEND\n"
            "END\nBEGIN SEED\nLOCATION 52 31\nDISPLACEMENT 1.5 -0.5\nEND\nEND\n")
    sf = SubsetFile(text=text)
    xy2, neigh2, seed2 = regular_grid(sf, 100, 80, 10, 11)
    # the seed goes first, at the grid point nearest its location; the snakes
    # start from it
    assert xy2[0].tolist() == [50.0, 30.0] and seed2[0] == 0 and neigh2[0] == -1
    assert sorted(map(tuple, xy2.tolist())) == sorted(map(tuple, xy.tolist()))
    assert neigh2[1] == 0


def test_oracle_vsg_matches_reference_gold():
    for k in FRAMES:
        g = _gold("dic_challenge_12_sorted", k)
        out, failed = O.vsg_strain(_fields(g), WINDOW)
        assert not failed.any()
        # the gold's displacements are printed to five digits: the strains
        # agree within that input rounding
        for col, gcol in ((0, 4), (1, 5)):
            assert np.all(np.abs(out[:, col] - g[:, gcol]) <= 2e-3 * np.abs(g[:, gcol]) + 5e-8), (k, col)


def test_oracle_vsg_exact_on_affine_fields_and_failures():
    ys, xs = np.mgrid[0:12, 0:15]
    x, y = 30.0 + 10 * xs.ravel(), 40.0 + 10 * ys.ravel()
    f = np.zeros((len(x), abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X], f[:, abi.F_COORD_Y] = x, y
    a, b, c, d = 0.0025, -0.001, 0.0015, 0.004
    f[:, abi.F_DISP_X] = 0.5 + a * (x - 100) + b * (y - 90)
    f[:, abi.F_DISP_Y] = -0.25 + c * (x - 100) + d * (y - 90)
    f[7, abi.F_SIGMA] = -1.0                       # a failed subset
    out, failed = O.vsg_strain(f, 45)
    ok = failed == 0
    assert failed[7] == 1 and ok.sum() == len(x) - 1
    # float inputs: the slopes are those of the rounded displacements
    assert np.max(np.abs(out[ok, 3] - a)) < 2e-6 and np.max(np.abs(out[ok, 6] - d)) < 2e-6
    gl_xx = 0.5 * (2 * a + a * a + c * c)
    assert np.max(np.abs(out[ok, 0] - gl_xx)) < 3e-6
    # an isolated point and a collinear neighbourhood fail
    g = np.zeros((4, abi.FIELD_STRIDE))
    g[:, abi.F_COORD_X] = [0, 10, 20, 500]
    g[:, abi.F_COORD_Y] = [0, 0, 0, 500]
    out, failed = O.vsg_strain(g, 50)
    assert failed.tolist() == [1, 1, 1, 1] and not out.any()


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _device_vsg(fields, window):
    from dice_b200.schema import Schema
    with Schema(abi.default_params()) as s:
        s.set_ref_image(np.zeros((64, 64), np.float32))
        s.set_fields(fields)
        out = s.vsg_strain(window)
        g = s.fields()
        assert s.device_status() == 0
    return out, g


@pytest.mark.gpu
def test_gpu_vsg_matches_oracle():
    _gpu()
    rng = np.random.default_rng(5)
    cases = [_fields(_gold("dic_challenge_12_sorted", k)) for k in FRAMES]
    # a scattered cloud with failed subsets and sparse corners
    n = 3000
    f = np.zeros((n, abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = np.round(rng.uniform(0, 2000, n))
    f[:, abi.F_COORD_Y] = np.round(rng.uniform(0, 1500, n))
    f[:, abi.F_DISP_X] = 1e-3 * f[:, abi.F_COORD_X] + rng.normal(0, 0.01, n)
    f[:, abi.F_DISP_Y] = -2e-3 * f[:, abi.F_COORD_Y] + rng.normal(0, 0.01, n)
    f[rng.random(n) < 0.05, abi.F_SIGMA] = -1.0
    cases.append(f)
    for fields, window in zip(cases, (WINDOW, WINDOW, WINDOW, 70)):
        want, failed = O.vsg_strain(fields, window)
        got, g = _device_vsg(fields, window)
        assert np.array_equal(g[:, abi.F_MATCH] == -1.0, (failed == 1) | (fields[:, abi.F_MATCH] == -1.0))
        ok = failed == 0
        assert np.allclose(got[:, :7], want, rtol=1e-6, atol=1e-12)
        assert (got[~ok, :7] == 0).all()
    assert (failed == 1).any() and (failed == 0).any()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["dic_challenge_12", "dic_challenge_12_sorted"])
def test_gpu_vsg_regression_files(tmp_path, variant):
    """The dic_challenge_12 result files rebuilt from their own displacement,
    gamma and match columns with the device's VSG strains, written in the
    reference's format and checked with DICe_Diff -t 0.05 -f 5.0E-5."""
    _gpu()
    p = abi.default_params(subset_size=27, enable_normal_strain=1)
    out = Output(p, fields=["COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X", "DISPLACEMENT_Y", "VSG_STRAIN_XX",
                            "VSG_STRAIN_YY", "GAMMA", "MATCH"], delimiter=",", omit_row_id=True,
                 ref_image="./images/oht_cfrp_00.tiff", step_size=(35, 35), strain_window=WINDOW,
                 sort_rows=variant.endswith("sorted"), initialization_method="USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY")
    grid = regular_grid(SubsetFile(text=str(GOLD["subset_file_dic_challenge_12"])), 400, 1040, 35, 27)[0]
    for k in FRAMES:
        g = _gold("dic_challenge_12", k)           # grid order
        assert np.array_equal(g[:, :2], grid)
        vsg, fields = _device_vsg(_fields(g), WINDOW)
        out.set_images(def_image="./images/oht_cfrp_%s.tiff" % k)
        out.write_frame(tmp_path, "DICe_solution", int(k), fields, vsg=vsg, first_frame=0, num_frames=11,
                        separate_files=False)
        n, rep = diff_text(str(GOLD["%s_gold_text_%s" % (variant, k)]),
                           open(tmp_path / ("DICe_solution_%s.txt" % k)).read(), tol=0.05, floor=5.0e-5)
        assert n == 0, rep


@pytest.mark.parametrize("variant", ["dic_challenge_12", "dic_challenge_12_sorted"])
def test_oracle_vsg_regression_files(tmp_path, variant):
    """The same files with the oracle's VSG (CPU)."""
    p = abi.default_params(subset_size=27, enable_normal_strain=1)
    out = Output(p, fields=["COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X", "DISPLACEMENT_Y", "VSG_STRAIN_XX",
                            "VSG_STRAIN_YY", "GAMMA", "MATCH"], delimiter=",", omit_row_id=True,
                 ref_image="./images/oht_cfrp_00.tiff", step_size=(35, 35), strain_window=WINDOW,
                 sort_rows=variant.endswith("sorted"), initialization_method="USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY")
    for k in FRAMES:
        g = _gold("dic_challenge_12", k)
        f = _fields(g)
        vsg = np.zeros((len(g), abi.VSG_STRIDE))
        vsg[:, :7] = O.vsg_strain(f, WINDOW)[0]
        out.set_images(def_image="./images/oht_cfrp_%s.tiff" % k)
        out.write_frame(tmp_path, "DICe_solution", int(k), f, vsg=vsg, first_frame=0, num_frames=11,
                        separate_files=False)
        n, rep = diff_text(str(GOLD["%s_gold_text_%s" % (variant, k)]),
                           open(tmp_path / ("DICe_solution_%s.txt" % k)).read(), tol=0.05, floor=5.0e-5)
        assert n == 0, rep


def _scattered(n, seed, fail_frac=0.05):
    rng = np.random.default_rng(seed)
    f = np.zeros((n, abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = np.round(rng.uniform(0, 600, n))
    f[:, abi.F_COORD_Y] = np.round(rng.uniform(0, 400, n))
    f[:, abi.F_DISP_X] = 1e-3 * f[:, abi.F_COORD_X] + rng.normal(0, 0.01, n)
    f[:, abi.F_DISP_Y] = -2e-3 * f[:, abi.F_COORD_Y] + rng.normal(0, 0.01, n)
    f[rng.random(n) < fail_frac, abi.F_SIGMA] = -1.0
    return f


def test_oracle_vsg_k_nearest_shells_equal_radius():
    """k nearest neighbourhoods (negative windows, the reference's knnSearch):
    on a square grid, k = 9 and k = 25 take whole shells of neighbours (self,
    4 + 4 at 1 and sqrt(2) steps; then 4 + 8 at 2 and sqrt(5), 4 at sqrt(8)),
    so they equal the radius windows that hold exactly those shells, bit for
    bit.  The nearest must be valid, as the reference tests neighbour 0."""
    ys, xs = np.mgrid[0:14, 0:17]
    x, y = 30.0 + 10 * xs.ravel(), 40.0 + 10 * ys.ravel()
    f = np.zeros((len(x), abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X], f[:, abi.F_COORD_Y] = x, y
    rng = np.random.default_rng(3)
    f[:, abi.F_DISP_X] = 0.5 + 0.0025 * (x - 100) + rng.normal(0, 1e-3, len(x))
    f[:, abi.F_DISP_Y] = -0.25 + 0.004 * (y - 90) + rng.normal(0, 1e-3, len(x))
    f[11, abi.F_SIGMA] = -1.0
    interior = (xs.ravel() >= 2) & (xs.ravel() <= 14) & (ys.ravel() >= 2) & (ys.ravel() <= 11)
    for k, window in ((9, 30), (25, 58)):   # radius 15 px: the 3 x 3 block; 29 px: the 5 x 5 block
        ok_k, fail_k = O.vsg_strain(f, -k)
        ok_r, fail_r = O.vsg_strain(f, window)
        assert np.array_equal(ok_k[interior], ok_r[interior])
        assert np.array_equal(fail_k[interior], fail_r[interior])
    out, failed = O.vsg_strain(f, -9)
    assert failed[11] == 1 and (failed == 0).sum() > 200
    assert np.max(np.abs(out[failed == 0, 3] - 0.0025)) < 1e-3
    with pytest.raises(AssertionError):
        O.vsg_strain(f[:5], -6)     # more neighbours than subsets


@pytest.mark.gpu
@pytest.mark.parametrize("k", [5, 9, 16, 40])
def test_gpu_vsg_k_nearest_matches_oracle(k):
    """The GPU's k nearest neighbourhoods (host lists, float squared distance,
    ties by index) equal the oracle's, and so do the fits, bit for bit, on a
    scattered cloud with failed subsets and on a square grid, where ties at
    the k-th distance are common."""
    _gpu()
    ys, xs = np.mgrid[0:20, 0:25]
    grid = np.zeros((xs.size, abi.FIELD_STRIDE))
    grid[:, abi.F_COORD_X], grid[:, abi.F_COORD_Y] = 5.0 + 7 * xs.ravel(), 9.0 + 7 * ys.ravel()
    grid[:, abi.F_DISP_X] = 1e-3 * grid[:, abi.F_COORD_X]
    grid[:, abi.F_DISP_Y] = 3e-3 * grid[:, abi.F_COORD_Y]
    grid[::13, abi.F_SIGMA] = -1.0
    for fields in (_scattered(2500, 11), grid):
        want, failed = O.vsg_strain(fields, -k)
        got, g = _device_vsg(fields, -k)
        assert np.array_equal(got[:, :7], want)
        assert np.array_equal(g[:, abi.F_MATCH] == -1.0, (failed == 1) | (fields[:, abi.F_MATCH] == -1.0))
        assert (failed == 0).any()
