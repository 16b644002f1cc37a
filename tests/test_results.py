"""Result writer (Output_Spec / Schema::write_output) and the DICe_Diff
comparator, and the reference's regression runs that use them.

The regression gold files of conformal_subset_def (five subsets, two
conformal, one obstructed and blocked) and simple_obstruction (37 frames of a
subset sliding under an obstruction) are checked the way the reference's
harness checks them: results written in its format, compared with
DICe_Diff -t 0.05 -f 5.0E-5 (tests/regression/CMakeLists.txt).  The
examples/obstruction run (tracking defaults with subset evolution) is checked
with the examples' own comparison, DICe_Diff -t 10.0 -f 1E-4
(tests/examples/CMakeLists.txt).  The oracle runs them here; the GPU runs
them in test_masks.py.
"""
import os
import subprocess

import numpy as np
import pytest

from dice_b200 import abi
from dice_b200 import synthetic as syn
from dice_b200.results import Output, diff_files, diff_text
from dice_b200.subset_file import SubsetFile
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = np.load(os.path.join(ROOT, "tests", "golden", "reference_gold.npz"))
DIFF_BIN = os.path.join(ROOT, "dice_b200", "bin", "dicegpu_diff")
REGRESSION_TOL, REGRESSION_FLOOR = 0.05, 5.0e-5
# "very loose tolerances for the examples (these are not regression tests)"
EXAMPLE_TOL, EXAMPLE_FLOOR = 10.0, 1.0e-4


def _row(**cols):
    r = np.zeros(abi.FIELD_STRIDE)
    for k, v in cols.items():
        r[getattr(abi, "F_" + k)] = v
    return r


def test_info_block_and_default_columns():
    p = abi.default_params(subset_size=27)
    o = Output(p, ref_image="ref.tif", def_image="def.tif")
    info = o.info_text().splitlines()
    assert info[0] == "***" and info[2] == "***" and info[-1] == "***"
    assert info[1].split()[1] == "Digital"                       # the masthead DICe_Diff skips
    assert info[3] == "*** Reference image: ref.tif "
    assert "*** Shape functions: Translation (u,v) " in info
    assert "*** Subset size: 27" in info and "*** Strain window: N/A" in info
    assert "*** Step size: x -1 y -1 (-1 implies not regular grid)" in info
    assert o.header_text("FRAME") == ("FRAME COORDINATE_X COORDINATE_Y DISPLACEMENT_X DISPLACEMENT_Y ROTATION_Z "
                                      "NORMAL_STRAIN_X NORMAL_STRAIN_Y SHEAR_STRAIN_XY SIGMA STATUS_FLAG\n")
    q = Output(abi.default_params(shape_function=abi.QUADRATIC_SF, enable_rotation=1))
    assert "NORMAL_STRAIN_X" not in q.header_text()
    assert "*** Shape functions: quadratic (A,B,C,D,E,F,G,H,I,J,K,L)" in q.info_text().splitlines()


def test_rows_round_to_float_and_print_4_4e():
    o = Output(abi.default_params(), fields="COORDINATE_X, DISPLACEMENT_X ,STATUS_FLAG,FIELD_3,SSSIG")
    r = _row(COORD_X=126.0, DISP_X=0.40060999, STATUS=1.0)
    unc = np.zeros(abi.UNCERTAINTY_STRIDE)
    unc[2] = 0.5
    assert o.row_text(7, r, unc) == "7 1.2600E+02 4.0061E-01 1.0000E+00 5.0000E-01 0.0000E+00\n"
    # a double whose digits change with the float conversion: printed as
    # the float the reference holds
    assert "%4.4E" % 1.00005 == "1.0001E+00" and "%4.4E" % float(np.float32(1.00005)) == "1.0000E+00"
    assert o.row_text(0, _row(DISP_X=1.00005)).split()[2] == "1.0000E+00"
    assert Output(abi.default_params(), fields=["GAMMA"], omit_row_id=True,
                  delimiter=",").row_text(3, _row(GAMMA=0.25)) == "2.5000E-01\n"
    with pytest.raises(RuntimeError):
        Output(abi.default_params(), fields="DISPLACEMENT_X,NOT_A_FIELD")
    with pytest.raises(RuntimeError):
        Output(abi.default_params(), fields="SIGMA,SIGMA")


def test_file_naming(tmp_path):
    o = Output(abi.default_params())
    f = np.zeros((12, abi.FIELD_STRIDE))
    f[:, abi.F_COORD_X] = np.arange(12)
    o.write_frame(tmp_path, "DICe_solution", 0, f)
    o.write_frame(tmp_path, "DICe_solution", 1, f)
    names = sorted(os.listdir(tmp_path))
    assert names[:3] == ["DICe_solution_00.txt", "DICe_solution_01.txt", "DICe_solution_02.txt"]
    assert len(names) == 12
    lines = open(tmp_path / "DICe_solution_11.txt").read().splitlines()
    assert lines[-3].startswith("FRAME ") and lines[-2].startswith("0 1.1000E+01") and lines[-1].startswith("1 ")
    o.write_frame(tmp_path, "frame", 7, f, first_frame=0, num_frames=100, separate_files=False)
    text = open(tmp_path / "frame_007.txt").read().splitlines()
    assert text[-13].startswith("SUBSET_ID ") and text[-1].startswith("11 ")


def test_diff_semantics():
    gold = "***\n*** Digital x\nFRAME A B\n0 1.0000E+00 2.0000E-05 0.0000E+00\n"
    same = "***\n*** Digital y\nFRAME A B\n0 1.0400E+00 9.0000E-05 1.0000E-09\n"
    assert diff_text(gold, same, tol=0.05, floor=5e-5)[0] == 0          # masthead, floor, tiny
    assert diff_text(gold, same, tol=0.05)[0] == 1                      # no floor: 2e-5 -> 9e-5 fails
    n, rep = diff_text(gold, "***\n*** Digital y\nFRAME A C\n0 1.0400E+00 2.0000E-05 0\n", tol=0.05)
    assert n == 1 and "[s]" in rep                                      # header strings compared
    assert diff_text(gold, "***\n*** Digital y\nFRAME A C\n0 1.0400E+00 2.0000E-05 0\n", tol=0.05,
                     numerical_only=True)[0] == 0
    assert diff_text(gold, "***\n*** Digital y\nFRAME A B\n", tol=0.05)[0] == 1   # result shorter than gold
    assert diff_text(gold, gold.replace("1.0000E+00", "1.0600E+00"), tol=0.05)[0] == 1
    assert diff_text("1,2,3\n", "1 2 3\n")[0] == 0                      # ',' and ' ' both delimit


def test_diff_cli(tmp_path):
    a, b = tmp_path / "a.txt", tmp_path / "b.txt"
    a.write_text("0 1.0000E+00\n")
    b.write_text("0 1.0300E+00\n")
    r = subprocess.run([DIFF_BIN, str(a), str(b), "-t", "0.05"], capture_output=True, text=True)
    assert r.returncode == 0 and "TEST PASSED" in r.stdout
    r = subprocess.run([DIFF_BIN, str(a), str(b), "-t", "0.01", "-v"], capture_output=True, text=True)
    assert r.returncode == 1 and "TEST FAILED" in r.stdout and "< 0" in r.stdout


def test_diff_parallel_pieces(tmp_path):
    (tmp_path / "serial.txt").write_text("HDR\n0 1.0 5.0\n1 2.0 6.0\n2 3.0 7.0\n")
    (tmp_path / "par.2.0.txt").write_text("HDR\n2 3.0 7.0\n0 1.0 5.0\n")
    (tmp_path / "par.2.1.txt").write_text("HDR\n1 2.0 6.04\n")
    # the parallel path of DICe_Diff compares |a - b| for a != 0
    assert diff_files(tmp_path / "serial.txt", tmp_path / "par", tol=0.05, num_procs=2)[0] == 0
    assert diff_files(tmp_path / "serial.txt", tmp_path / "par", tol=0.01, num_procs=2)[0] == 1
    (tmp_path / "par.2.1.txt").write_text("HDR\n")
    assert diff_files(tmp_path / "serial.txt", tmp_path / "par", tol=0.05, num_procs=2)[0] == 1


def conformal_subset_def_case():
    """The conformal_subset_def regression: subsets, params, images."""
    sf = SubsetFile(text=str(GOLD["subset_file_conformal_subset_def"]), width=512, height=512)
    p = abi.default_params(subset_size=27, correlation_routine=abi.TRACKING_ROUTINE, use_def_gradients=0)
    ref = GOLD["ref_speckled"].astype(np.float32)
    deff = GOLD["def_speckled"].astype(np.float32)
    out = Output(p, ref_image="../../component/images/refSpeckled.tif",
                 def_image="../../component/images/defSpeckled.tif")
    return sf, p, ref, deff, out


def simple_obstruction_case():
    sf = SubsetFile(text=str(GOLD["subset_file_simple_obstruction"]), width=200, height=200)
    p = abi.tracking_default_params(subset_size=-1, use_def_gradients=0, normalize_gamma_with_active_pixels=1)
    out = Output(p, fields=["COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X"], ref_image="./images/Img_00.tif",
                 def_image="./images/Img_00.tif")
    return sf, p, GOLD["simple_obstruction_frames"], out


def obstruction_example_case():
    """examples/obstruction: a conformal subset (polygon boundary, an excluded
    and an obstructed rectangle) rotating 2 degrees per frame about (100, 100)
    behind a static bar, blocked by a 17 x 17 subset; params.xml sets the
    tracking defaults (subset evolution on), bilinear interpolation, simplex
    and disp_jump_tol 5.  Its gold rows FRAME r = 1..11 are the images
    obstruction_{r+1} against obstruction_01 (subset 1 reproduces them to the
    printed digits)."""
    sf = SubsetFile(text=str(GOLD["subset_file_obstruction_example"]), width=200, height=200)
    p = abi.tracking_default_params(subset_size=-1, use_def_gradients=0, interpolation=abi.BILINEAR,
                                    disp_jump_tol=5.0)
    out = Output(p, fields=["COORDINATE_X", "COORDINATE_Y", "ROTATION_Z", "SIGMA", "GAMMA"], delimiter=",",
                 ref_image="./images/obstruction_01.tif", def_image="./images/obstruction_01.tif")
    return sf, p, GOLD["obstruction_example_frames"].astype(np.float32), out


def oracle_obstruction_example(p, sf, frames):
    """The oracle over the example's frames: field rows and evolution state
    (state, reference values) after each frame."""
    f = syn.init_fields(sf.coordinates[:, 0], sf.coordinates[:, 1])
    offs, ids = blocking_csr(sf)
    evo, rows, states = {}, [], []
    for k in range(1, len(frames)):
        O.execute_frame_shapes(p, frames[0], frames[k], f, sf.shapes, sf.vx, sf.vy, offs, ids,
                               force_simplex=sf.force_simplex, first_frame=(k == 1), evolution=evo,
                               frame_index=k - 1)
        rows.append(f.copy())
        if evo:
            states.append((evo["flag"].copy(), evo["f"].copy()))
    return rows, states


def check_example_files(tmp_path, out, rows):
    """Per-subset files (separate_output_file_for_each_subset) against the
    example's gold: (failed lines at the example tolerance, at the
    regression tolerance) per subset."""
    for k, f in enumerate(rows):
        out.write_frame(tmp_path, "DICe_solution", k + 1, f, first_frame=1, num_frames=len(rows),
                        separate_files=True)
    res = []
    for i in range(2):
        text = str(GOLD["obstruction_example_gold_text_%d" % i])
        got = open(tmp_path / ("DICe_solution_%d.txt" % i)).read()
        res.append((diff_text(text, got, tol=EXAMPLE_TOL, floor=EXAMPLE_FLOOR)[0],
                    diff_text(text, got, tol=REGRESSION_TOL, floor=REGRESSION_FLOOR)[0]))
    return res


def blocking_csr(sf):
    offs = np.zeros(len(sf.blocking) + 1, np.int32)
    ids = []
    for i, b in enumerate(sf.blocking):
        ids += list(b)
        offs[i + 1] = offs[i] + len(b)
    return offs, np.asarray(ids, np.int32)


def check_against_gold(tmp_path, out, rows_per_frame, gold_texts):
    """Writes the frames' field rows in the reference's format and runs the
    reference's regression comparison on every gold file."""
    for k, f in enumerate(rows_per_frame):
        out.write_frame(tmp_path, "DICe_solution", k, f)
    for i, text in enumerate(gold_texts):
        result = open(tmp_path / ("DICe_solution_%d.txt" % i)).read()
        n, rep = diff_text(text, result, tol=REGRESSION_TOL, floor=REGRESSION_FLOOR)
        assert n == 0, rep


def test_oracle_conformal_subset_def_gold(tmp_path):
    sf, p, ref, deff, out = conformal_subset_def_case()
    f = syn.init_fields(sf.coordinates[:, 0], sf.coordinates[:, 1])
    offs, ids = blocking_csr(sf)
    O.execute_frame_shapes(p, ref, deff, f, sf.shapes, sf.vx, sf.vy, offs, ids, force_simplex=sf.force_simplex)
    check_against_gold(tmp_path, out, [f], [str(GOLD["conformal_subset_def_gold_text_%d" % k]) for k in range(5)])
    # the Gauss-Newton subsets (1, 2) agree to the printed digits; the
    # simplex ones (blocked / blocking, forced) stop on the flat valley of
    # gamma where rounding decides the stopping iteration
    gold = GOLD["conformal_subset_def_gold"]
    assert np.max(np.abs(f[[1, 2], abi.F_DISP_X] - gold[[1, 2], 3])) < 1e-5
    assert np.array_equal(f[:, abi.F_STATUS], gold[:, 10])


def test_oracle_simple_obstruction_gold(tmp_path):
    sf, p, frames, out = simple_obstruction_case()
    f = syn.init_fields(sf.coordinates[:, 0], sf.coordinates[:, 1])
    rows, active = [], []
    for k in range(frames.shape[0]):
        O.execute_frame_shapes(p, frames[0].astype(np.float32), frames[k].astype(np.float32), f, sf.shapes, sf.vx,
                               sf.vy, first_frame=(k == 0))
        rows.append(f.copy())
        active.append(f[0, abi.F_ACTIVE_PIXELS])
    check_against_gold(tmp_path, out, rows, [str(GOLD["simple_obstruction_gold_text"])])
    # the subset slides under the obstruction: its active pixels shrink
    assert active[0] == 75 * 29 and active[-1] < 200 and np.all(np.diff(active) <= 0)


def test_oracle_obstruction_example_with_subset_evolution(tmp_path):
    sf, p, frames, out = obstruction_example_case()
    assert p.use_subset_evolution == 1 and p.correlation_routine == abi.TRACKING_ROUTINE
    rows, states = oracle_obstruction_example(p, sf, frames)
    res = check_example_files(tmp_path, out, rows)
    # both files pass the example's comparison; the blocking subset (no
    # excluded pixels, Gauss-Newton-free 17 x 17 square) matches its gold at
    # the regression tolerance too
    assert res[0][0] == 0 and res[1] == (0, 0), res
    # the first two frames turn nothing on (frame_id_ > first_frame_id_ +
    # frame_skip_); the excluded pixels that rotate out from under the bar do
    # later, with image intensities as their references
    # (36 of the subset's 4430 pixels are excluded)
    flag0 = states[0][0]
    assert (flag0 == 0).sum() == 36 and not (states[0][0] == 2).any() and not (states[1][0] == 2).any()
    on = [(st == 2).sum() for st, _ in states]
    assert on[-1] >= 5 and all(b >= a for a, b in zip(on, on[1:]))
    last_state, last_f = states[-1]
    assert np.all((last_f[last_state == 2] >= 0) & (last_f[last_state == 2] <= 255))
    assert (last_f[last_state != 2] == 0).all()
    # the turned-on pixels join the count of active pixels
    n0 = sf.coordinates.shape[0]
    assert n0 == 2 and rows[-1][1, abi.F_ACTIVE_PIXELS] == 289


def test_oracle_subset_evolution_is_frame_local_in_generic_routine():
    """The generic routine rebuilds its objectives every frame
    (DICe_Schema.cpp:1708-1724): evolution leaves no state behind."""
    sf, p, frames, _ = obstruction_example_case()
    p.correlation_routine = abi.GENERIC_ROUTINE
    sub = frames[:5]
    rows_on, states = oracle_obstruction_example(p, sf, sub)
    p.use_subset_evolution = 0
    rows_off, _ = oracle_obstruction_example(p, sf, sub)
    assert not states
    for a, b in zip(rows_on, rows_off):
        assert np.array_equal(a, b)
