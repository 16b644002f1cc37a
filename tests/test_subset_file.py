"""Subset-file parser (read_subset_file / read_shapes, DICe_Parser.cpp:1098-1860).

The reference's own subset files (committed as text in the golden fixtures)
are parsed and every value is checked against the file's content; the
malformed inputs the reference rejects are rejected with a message.
"""
import os

import numpy as np
import pytest

from dice_b200 import abi
from dice_b200.subset_file import SubsetFile, SubsetFileError, FEATURE_SKIP_SOLVE, SEED_DISPLACEMENT, SEED_ROTATION

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_gold.npz"))


def _text(name):
    return str(GOLD["subset_file_" + name])


def _poly(sf, shape):
    o, n = shape.vertex_offset, shape.vertex_count
    return list(zip(sf.vx[o:o + n].tolist(), sf.vy[o:o + n].tolist()))


def test_conformal_subset_def_file():
    sf = SubsetFile(text=_text("conformal_subset_def"), width=512, height=512)
    assert sf.info.n_subsets == 5 and sf.info.n_conformal == 2 and sf.info.region_of_interest == 0
    # comment rows, a comment after a number and blank rows are skipped
    assert sf.coordinates.tolist() == [[126, 157], [125, 250], [397, 139], [177, 314], [395, 405]]
    s2 = [s for s in sf.shapes if s.subset == 2]
    assert [(s.kind, s.role) for s in s2] == [(abi.SHAPE_POLYGON, 0), (abi.SHAPE_CIRCLE, 0), (abi.SHAPE_POLYGON, 0)]
    assert _poly(sf, s2[0]) == [(307, 136), (352, 86), (426, 109), (421, 243), (372, 143)]
    assert (s2[1].cx, s2[1].cy, s2[1].radius) == (362, 201, 45.0)
    assert _poly(sf, s2[2]) == [(359, 228), (455, 175), (437, 267)]
    s3 = [s for s in sf.shapes if s.subset == 3]
    assert [(s.kind, s.role) for s in s3] == [(abi.SHAPE_CIRCLE, 0), (abi.SHAPE_POLYGON, abi.ROLE_EXCLUDED),
                                            (abi.SHAPE_POLYGON, abi.ROLE_OBSTRUCTED)]
    assert (s3[0].cx, s3[0].cy, s3[0].radius) == (178, 352, 64.0)
    assert _poly(sf, s3[1]) == [(148, 341), (160, 374), (205, 340)]
    assert _poly(sf, s3[2]) == [(130, 423), (252, 366), (266, 402), (148, 460)]
    assert sf.blocking == [[], [], [], [0, 4], []]
    assert not sf.force_simplex.any() and not sf.seed_flags.any() and not sf.features.any()


def test_obstruction_and_mechanism_files():
    sf = SubsetFile(text=_text("simple_obstruction"), width=200, height=200)
    assert sf.coordinates.tolist() == [[64, 100]]
    assert [(s.kind, s.role, s.cx, s.cy, s.width, s.height) for s in sf.shapes] == [
        (abi.SHAPE_RECTANGLE, 0, 64, 100, 75, 29), (abi.SHAPE_RECTANGLE, abi.ROLE_OBSTRUCTED, 149, 104, 93, 109)]
    ex = SubsetFile(text=_text("obstruction_example"))
    assert ex.blocking == [[1], []]
    roles = [(s.subset, s.kind, s.role) for s in ex.shapes]
    assert roles == [(0, abi.SHAPE_POLYGON, 0), (0, abi.SHAPE_RECTANGLE, 1), (0, abi.SHAPE_RECTANGLE, 2),
                     (1, abi.SHAPE_RECTANGLE, 0)]
    assert len(_poly(ex, ex.shapes[0])) == 13
    mech = SubsetFile(text=_text("mechanism"))
    assert mech.info.n_subsets == 4 and mech.info.n_conformal == 4
    kinds = [(s.subset, s.kind) for s in mech.shapes]
    assert kinds == [(0, abi.SHAPE_POLYGON), (0, abi.SHAPE_POLYGON), (1, abi.SHAPE_RECTANGLE),
                     (2, abi.SHAPE_CIRCLE), (3, abi.SHAPE_RECTANGLE)]
    skip = SubsetFile(text=_text("mechanism_skip_solves"))
    # subset 0 reads its frame ids from another file (not read here: an
    # unsupported feature); subset 1 lists them on the line
    assert skip.features.tolist() == [FEATURE_SKIP_SOLVE, 0]
    assert skip.skip_solve == [None, [4903, 4912, 4915]]
    # frame_should_be_skipped: solving starts on; each id toggles it
    assert [skip.skip_solve_flags(fr)[1] for fr in (4900, 4903, 4911, 4912, 4914, 4915, 5000)] == [0, 1, 1, 0, 0, 1, 1]
    assert not SubsetFile(text=_text("mechanism_optical_flow")).features.any()


def test_seeds_force_simplex_and_rectangle_corners():
    text = """
    BEGIN SUBSET_COORDINATES
      20 30
      40 50
    END
    begin conformal_subset
      subset_id 1
      begin boundary
        begin rectangle
          upper_left 30 40
          lower_right 51 61
        end
      end
      begin seed
        displacement 1.5 -2.25
        rotation 0.125
      end
      force_simplex
    end
    """
    sf = SubsetFile(text=text, width=100, height=100)
    r = sf.shapes[0]
    # width = lr - ul, centre = width / 2 + ul (read_rectangle)
    assert (r.subset, r.cx, r.cy, r.width, r.height) == (1, 40, 50, 21, 21)
    assert sf.force_simplex.tolist() == [0, 1]
    assert sf.seed_flags.tolist() == [0, SEED_DISPLACEMENT | SEED_ROTATION]
    assert sf.seed_values[1].tolist() == [1.5, -2.25, 0.0, 0.0, 0.0, 0.125]


@pytest.mark.parametrize("text, why", [
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nBEGIN BOUNDARY\nBEGIN CIRCLE\nCENTER 10 20\n"
     "RADIUS 3\nEND\nEND\nEND\n", "subset id"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\nBEGIN BOUNDARY\nBEGIN POLYGON\n"
     "BEGIN VERTICES\n1 2\n3 4\nEND\nEND\nEND\nEND\n", "three vertices"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\nBEGIN BOUNDARY\nBEGIN CIRCLE\n"
     "CENTER 10 20\nEND\nEND\nEND\n", "incomplete circle"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\nBEGIN BOUNDARY\nBEGIN ELLIPSE\n"
     "END\nEND\nEND\n", "unrecognized shape"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\nBEGIN BOUNDARY\nBEGIN RECTANGLE\n"
     "UPPER_LEFT 10 10\nLOWER_RIGHT 5 20\nEND\nEND\nEND\n", "inverted"),
    ("BEGIN SUBSET_COORDINATES\n10 # 20\nEND\n", "not enough values"),
    ("BEGIN SUBSET_COORDINATES\n10 220\nEND\n", "coordinate y"),
    ("BEGIN SUBSET_COORDINATES\nEND\n", "no subset coordinates"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\nTEST_FOR_MOTION\nBEGIN BOUNDARY\n"
     "BEGIN CIRCLE\nCENTER 10 20\nRADIUS 3\nEND\nEND\nEND\n", "motion window"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN REGION_OF_INTEREST\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\n"
     "BEGIN BOUNDARY\nBEGIN CIRCLE\nCENTER 10 20\nRADIUS 3\nEND\nEND\nEND\n", "region of interest"),
    ("BEGIN SUBSET_COORDINATES\n10 20\nEND\nBEGIN CONFORMAL_SUBSET\nSUBSET_ID 0\nFOO\nEND\n", "unknown block"),
])
def test_malformed_files_are_rejected(text, why):
    with pytest.raises(SubsetFileError) as e:
        SubsetFile(text=text, width=100, height=100)
    assert why in str(e.value)


def test_crlf_lines_integer_bases_and_first_definition_wins():
    text = ("BEGIN SUBSET_COORDINATES\r\n 10 20\r\n 30 40\r\nEND\r\n"
            "BEGIN CONFORMAL_SUBSET\r\nSUBSET_ID 1\r\nBEGIN BOUNDARY\r\nBEGIN CIRCLE\r\nCENTER 010 20\r\nRADIUS 4\r\n"
            "END\r\nEND\r\nEND\r\n"
            "BEGIN CONFORMAL_SUBSET\nSUBSET_ID 1\nBEGIN BOUNDARY\nBEGIN CIRCLE\nCENTER 30 40\nRADIUS 9\nEND\nEND\nEND\n")
    sf = SubsetFile(text=text)
    assert sf.coordinates.tolist() == [[10, 20], [30, 40]]
    # strtol base 0 reads "010" as octal; a repeated id keeps its first definition
    assert [(s.cx, s.cy, s.radius) for s in sf.shapes] == [(8, 20, 4.0)]


def test_missing_file_reports_path():
    with pytest.raises(SubsetFileError) as e:
        SubsetFile(path="/nonexistent/subsets.txt")
    assert "does not exist" in str(e.value)
