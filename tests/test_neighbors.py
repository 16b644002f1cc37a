"""Neighbour initialization (USE_NEIGHBOR_VALUES, _FIRST_STEP_ONLY).

Field_Value_Initializer::initial_guess (DICe_Initializer.cpp:398-436) takes a
subset's initial guess from its NEIGHBOR_ID's field values; the reference
runs the subsets in index order, so a chain of neighbours carries a seed's
solution across a displacement too large for a zero start.  The oracle
restates the rule; the GPU (dependency waves, chains as one sequential
launch, a reverse chain in one wave reading frame-start values) equals it,
and a captured two-frame sequence equals the frame calls.
"""
import numpy as np
import pytest
import torch

from dice_b200 import abi
from dice_b200 import synthetic as syn
from dice_b200.subset_file import SubsetFile, regular_grid
from oracle import oracle as O
from tests._exact import assert_rows_equal

W, H = 200, 160
U, V = 9.7, -7.4          # beyond the Gauss-Newton capture range from a zero start
SEEDED = ("BEGIN REGION_OF_INTEREST\nBEGIN BOUNDARY\nBEGIN RECTANGLE\nCENTER 100 80\nWIDTH 200\nHEIGHT 160\n"
          "END\nEND\nBEGIN SEED\nLOCATION 100 80\nDISPLACEMENT %g %g\nEND\nEND\n" % (U, V))


def _images():
    ref = syn.speckle_image(W, H, seed=31, blur_sigma=0.8)
    f1 = syn.warp_image(ref, lambda X, Y: (torch.full_like(X, U), torch.full_like(Y, V)), noise_sigma=0.5, seed=7)
    f2 = syn.warp_image(ref, lambda X, Y: (torch.full_like(X, U + 0.4), torch.full_like(Y, V - 0.3)),
                        noise_sigma=0.5, seed=8)
    return ref.numpy(), f1.numpy(), f2.numpy()


def _grid(seeded):
    sf = SubsetFile(text=SEEDED) if seeded else None
    xy, neigh, seed = regular_grid(sf, W, H, 12, 21)
    f = syn.init_fields(xy[:, 0], xy[:, 1])
    f[seed >= 0, abi.F_DISP_X] = U
    f[seed >= 0, abi.F_DISP_Y] = V
    if not seeded:                     # the chains' first points carry the start
        f[neigh < 0, abi.F_DISP_X] = U
        f[neigh < 0, abi.F_DISP_Y] = V
    return f, neigh


def _params(method, **kw):
    return abi.default_params(subset_size=21, optimization=abi.GRADIENT_BASED, initialization_method=method,
                              fast_solver_tolerance=1e-5, **kw)


def test_oracle_neighbor_chain_carries_the_seed():
    ref, f1, _ = _images()
    for seeded in (False, True):
        f, neigh = _grid(seeded)
        g = f.copy()
        O.execute_frame(_params(abi.USE_NEIGHBOR_VALUES), ref, f1, g, neighbors=neigh)
        ok = g[:, abi.F_SIGMA] >= 0
        assert ok.mean() > 0.95
        assert np.max(np.abs(g[ok, abi.F_DISP_X] - U)) < 0.05 and np.max(np.abs(g[ok, abi.F_DISP_Y] - V)) < 0.05
        has = (neigh >= 0) & (neigh != np.arange(len(neigh)))
        assert (g[has & ok, abi.F_STATUS] == 3).all() and (g[~has & ok, abi.F_STATUS] == 1).all()
        # the same grid from field values: the zero starts do not reach the solution
        h = f.copy()
        O.execute_frame(_params(abi.USE_FIELD_VALUES), ref, f1, h, neighbors=neigh)
        good = (h[:, abi.F_SIGMA] >= 0) & (np.abs(h[:, abi.F_DISP_X] - U) < 0.05)
        assert good.mean() < 0.2


def test_oracle_first_step_only_and_index_order():
    ref, f1, f2 = _images()
    f, neigh = _grid(False)
    p = _params(abi.USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY)
    O.execute_frame(p, ref, f1, f, first_frame=True, neighbors=neigh)
    assert (f[neigh >= 0, abi.F_STATUS] == 3).all()
    O.execute_frame(p, ref, f2, f, first_frame=False, neighbors=neigh)
    ok = f[:, abi.F_SIGMA] >= 0
    assert (f[ok, abi.F_STATUS] == 1).all() and np.max(np.abs(f[ok, abi.F_DISP_X] - U - 0.4)) < 0.05
    # a reverse chain: every neighbour has a higher index, so each start is
    # the neighbour's frame-start row (zeros): the chain does not carry
    g, _ = _grid(False)
    rev = np.append(np.arange(1, len(g)), -1).astype(np.int32)
    g[0, abi.F_DISP_X] = g[0, abi.F_DISP_Y] = 0.0
    g[-1, abi.F_DISP_X], g[-1, abi.F_DISP_Y] = U, V
    O.execute_frame(_params(abi.USE_NEIGHBOR_VALUES), ref, f1, g, neighbors=rev)
    good = (g[:, abi.F_SIGMA] >= 0) & (np.abs(g[:, abi.F_DISP_X] - U) < 0.05)
    assert good[-1] and good[-2] and good.mean() < 0.2


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _device(p, ref, frames, f, neigh, capture=False):
    from dice_b200.schema import Schema
    rows = []
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        s.set_neighbors(neigh)
        for d in frames:
            s.set_def_image(d)
            s.execute_correlation()
            rows.append(s.fields())
        if capture:
            s.capture_sequence([torch.from_numpy(d).cuda() for d in frames], reset_fields=torch.from_numpy(f).cuda())
            s.launch_sequence()
            torch.cuda.synchronize()
            assert np.array_equal(s.fields(), rows[-1])
        assert s.device_status() == 0
    return rows


def _compare(got, want):
    assert_rows_equal(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["chain", "seeded_tree", "reverse", "quadratic"])
def test_gpu_neighbor_initialization_matches_oracle(case):
    _need_gpu()
    ref, f1, _ = _images()
    f, neigh = _grid(case == "seeded_tree")
    p = _params(abi.USE_NEIGHBOR_VALUES)
    if case == "reverse":
        neigh = np.append(np.arange(1, len(f)), -1).astype(np.int32)
        f[0, abi.F_DISP_X] = f[0, abi.F_DISP_Y] = 0.0
        f[-1, abi.F_DISP_X], f[-1, abi.F_DISP_Y] = U, V
    if case == "quadratic":
        p = _params(abi.USE_NEIGHBOR_VALUES, shape_function=abi.QUADRATIC_SF)
        f = syn.init_fields(f[:, abi.F_COORD_X], f[:, abi.F_COORD_Y], quadratic=True)
        f[neigh < 0, abi.F_QUAD_A + 5] = U
        f[neigh < 0, abi.F_QUAD_A + 11] = V
    want = f.copy()
    O.execute_frame(p, ref, f1, want, neighbors=neigh)
    got = _device(p, ref, [f1], f, neigh)[0]
    _compare(got, want)
    if case in ("chain", "seeded_tree"):
        assert (want[:, abi.F_SIGMA] >= 0).mean() > 0.95
    if case == "quadratic":
        # a subset that fails fails every later one on its chain
        # (INITIALIZE_FAILED from the neighbour's sigma of -1)
        assert ((want[:, abi.F_STATUS] == 3) & (want[:, abi.F_SIGMA] >= 0)).sum() > 40
        assert (want[:, abi.F_STATUS] == 5).any()


@pytest.mark.gpu
def test_gpu_first_step_only_sequence_and_graph():
    _need_gpu()
    ref, f1, f2 = _images()
    f, neigh = _grid(True)
    p = _params(abi.USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY)
    want = f.copy()
    O.execute_frame(p, ref, f1, want, first_frame=True, neighbors=neigh)
    w1 = want.copy()
    O.execute_frame(p, ref, f2, want, first_frame=False, neighbors=neigh)
    rows = _device(p, ref, [f1, f2], f, neigh, capture=True)
    _compare(rows[0], w1)
    _compare(rows[1], want)


# ---- the reference's regressions ---------------------------------------------
# parallel_seed_first_step_only (two frames) and parallel_subsets_seed (one):
# four seeded 50 x 50 regions of interest on the speckled pair, step 10,
# subset 27, neighbour initialization from the seeds along the grid's snakes,
# Keys-4, GRADIENT_BASED_THEN_SIMPLEX, translation only, file-fed images
# (reference gradients).  Checked with DICe_Diff -t 0.05 -f 5.0E-5.
SEED_REGRESSIONS = {"parallel_seed_first_step_only": (abi.USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY, 2),
                    "parallel_subsets_seed": (abi.USE_NEIGHBOR_VALUES, 1)}


def _seed_regression(name):
    from test_results import GOLD
    method, nframes = SEED_REGRESSIONS[name]
    sf = SubsetFile(text=str(GOLD["subset_file_" + name]))
    p = abi.default_params(subset_size=27, initialization_method=method, use_def_gradients=0)
    from dice_b200.results import Output
    out = Output(p, fields=["COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X", "DISPLACEMENT_Y", "SIGMA"],
                 ref_image="../../component/images/refSpeckled.tif", step_size=(10, 10),
                 initialization_method=["USE_FIELD_VALUES", "USE_NEIGHBOR_VALUES",
                                        "USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY"][method])
    ref = GOLD["ref_speckled"].astype(np.float32)
    deff = GOLD["def_speckled"].astype(np.float32)
    golds = [str(GOLD["%s_gold_text_%d" % (name, k)]) for k in range(nframes)]
    return sf, p, out, ref, deff, golds


def _check_seed_files(tmp_path, out, rows, golds):
    from test_results import REGRESSION_FLOOR, REGRESSION_TOL
    from dice_b200.results import diff_text
    for k, (r, gold) in enumerate(zip(rows, golds)):
        # the second frame correlates a copy of the deformed image
        out.set_images(def_image="../../component/images/%s.tif" % ("defSpeckled" if k == 0 else "defSpeckledCopy"))
        out.write_frame(tmp_path, "DICe_solution", k, r, first_frame=0, num_frames=len(rows), separate_files=False)
        n, rep = diff_text(gold, open(tmp_path / ("DICe_solution_%d.txt" % k)).read(), tol=REGRESSION_TOL,
                           floor=REGRESSION_FLOOR)
        assert n == 0, rep


@pytest.mark.parametrize("name", sorted(SEED_REGRESSIONS))
def test_oracle_seed_regressions(tmp_path, name):
    sf, p, out, ref, deff, golds = _seed_regression(name)
    xy, neigh, seed = regular_grid(sf, 512, 512, 10, 27)
    f = syn.init_fields(xy[:, 0], xy[:, 1])
    f[seed >= 0, abi.F_DISP_X] = 0.4      # the regions' seeds
    f[seed >= 0, abi.F_DISP_Y] = 0.4
    rows = []
    for k in range(len(golds)):
        O.execute_frame(p, ref, deff, f, first_frame=(k == 0), neighbors=neigh)
        rows.append(f.copy())
    # 4 seeds start from their own rows, the other 60 from their neighbours
    assert (rows[0][:, abi.F_STATUS] == 3).sum() == 60
    _check_seed_files(tmp_path, out, rows, golds)


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(SEED_REGRESSIONS))
def test_gpu_seed_regressions(tmp_path, name):
    _need_gpu()
    from dice_b200.schema import Schema
    sf, p, out, ref, deff, golds = _seed_regression(name)
    rows = []
    with Schema(p) as s:
        s.set_ref_image(ref)
        sf.apply_grid(s, 512, 512, 10)    # grid, seeds and neighbours
        for _ in golds:
            s.set_def_image(deff)
            s.execute_correlation()
            rows.append(s.fields())
        assert s.device_status() == 0
    assert (rows[0][:, abi.F_STATUS] == 3).sum() == 60
    _check_seed_files(tmp_path, out, rows, golds)


def test_oracle_rejects_other_initializers():
    """Phase correlation, optical flow, feature matching and the other
    initializers are outside the path: DICEGPU_ERR_UNSUPPORTED."""
    ref, f1, _ = _images()
    f, neigh = _grid(False)
    for method in (3, 4, 5, 6):
        with pytest.raises(RuntimeError, match=str(abi.ERR_UNSUPPORTED)):
            O.execute_frame(_params(method), ref, f1, f.copy(), neighbors=neigh)


def test_abi_rejects_other_initializers():
    """dicegpu_create validates the params before any device call."""
    import ctypes
    lib = abi.load_library()
    ctx = ctypes.c_void_p()
    for method in (3, 4, 5, 6):
        assert lib.dicegpu_create(ctypes.byref(_params(method)), ctypes.byref(ctx)) == abi.ERR_UNSUPPORTED
