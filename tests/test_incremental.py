"""Incremental formulation (use_incremental_formulation).

Each frame after the first of a sequence correlates against the previous
deformed frame (DICe_Main.cpp:324-328, Schema::set_ref_image(prev_img())),
starts with DISPLACEMENT_X / _Y at 0 and ends with them accumulated; the
first frame of the sequence is not accumulated (DICe_Schema.cpp:1671-1675,
1775-1789).  The oracle runs the rule over a translating speckle sequence;
the GPU equals it frame by frame, and a captured sequence (reference
restored at each replay, the new reference taken from the previous frame on
the device) equals the frame-by-frame calls bit for bit.
"""
import numpy as np
import pytest
import torch

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O
from tests._exact import assert_rows_equal

STEP = (0.35, -0.25)     # px per frame


def _case(first_shift=0):
    ref = syn.speckle_image(192, 160, seed=21, blur_sigma=0.8)
    frames = [syn.warp_image(ref, lambda X, Y, k=k: (torch.full_like(X, STEP[0] * k),
                                                     torch.full_like(Y, STEP[1] * k)),
                             noise_sigma=0.5, seed=100 + k).numpy()
              for k in range(first_shift, first_shift + 5)]
    cx, cy = syn.grid_points(192, 160, 21, 16)
    p = abi.default_params(subset_size=21, use_incremental_formulation=1, optimization=abi.GRADIENT_BASED,
                           fast_solver_tolerance=1e-5)
    return ref.numpy(), frames, cx, cy, p


def test_oracle_incremental_accumulates_the_increments():
    ref, frames, cx, cy, p = _case()
    rows = O.execute_sequence(p, ref, frames, syn.init_fields(cx, cy))
    for k, f in enumerate(rows):
        assert (f[:, abi.F_STATUS] >= 0).all()
        assert np.max(np.abs(f[:, abi.F_DISP_X] - STEP[0] * k)) < 0.02, k
        assert np.max(np.abs(f[:, abi.F_DISP_Y] - STEP[1] * k)) < 0.02, k
    # the same sequence against the fixed reference gives the same totals
    p.use_incremental_formulation = 0
    direct = O.execute_sequence(p, ref, frames, syn.init_fields(cx, cy))
    assert np.max(np.abs(direct[-1][:, abi.F_DISP_X:abi.F_DISP_Y + 1] -
                         rows[-1][:, abi.F_DISP_X:abi.F_DISP_Y + 1])) < 0.02


def test_oracle_incremental_first_frame_not_accumulated():
    """A sequence whose first frame is already displaced: its displacement
    is reported at that frame and left out of the later totals (the
    accumulation starts at frame_id_ > first_frame_id_)."""
    ref, frames, cx, cy, p = _case(first_shift=1)
    rows = O.execute_sequence(p, ref, frames, syn.init_fields(cx, cy))
    assert np.max(np.abs(rows[0][:, abi.F_DISP_X] - STEP[0])) < 0.02
    # frame k (k >= 1) holds the increments of frames 1..k only
    for k in range(1, len(rows)):
        assert np.max(np.abs(rows[k][:, abi.F_DISP_X] - STEP[0] * k)) < 0.02, k


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
@pytest.mark.parametrize("first_shift", [0, 1])
def test_gpu_incremental_matches_oracle(first_shift):
    _need_gpu()
    from dice_b200.schema import Schema
    ref, frames, cx, cy, p = _case(first_shift)
    f0 = syn.init_fields(cx, cy)
    want = O.execute_sequence(p, ref, frames, f0.copy())
    rows = []
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f0)
        for k, d in enumerate(frames):
            if k > 0:
                s.set_ref_from_def()
            s.set_def_image(d)
            s.execute_correlation()
            rows.append(s.fields())
        assert s.device_status() == 0
        # the sequence as one CUDA graph, replayed twice: each replay starts
        # from the reference it was captured with
        s.set_ref_image(ref)
        s.capture_sequence([torch.from_numpy(d).cuda() for d in frames], reset_fields=torch.from_numpy(f0).cuda())
        for _ in range(2):
            s.launch_sequence()
            torch.cuda.synchronize()
            assert np.array_equal(s.fields(), rows[-1])
        assert s.device_status() == 0
    for k in range(len(rows)):
        assert_rows_equal(rows[k], want[k])


# ---- the reference's incremental regression ----------------------------------
# tests/regression/incremental: one 39 x 39 subset at (42, 42), all six affine
# parameters, Keys-4, Gauss-Newton, reference image defSyntheticSpeckled0 and
# frames 0..5 shifted by 1 px per frame; the result file of frame k reports
# the previous frame as its reference image.  DICe_Diff -t 0.05 -f 5.0E-5.
def _incremental_regression():
    from test_results import GOLD
    from dice_b200.results import Output
    frames = [GOLD["def_synthetic_%d" % k].astype(np.float32) for k in range(6)]
    p = abi.default_params(subset_size=39, interpolation=abi.KEYS_FOURTH, optimization=abi.GRADIENT_BASED,
                           use_incremental_formulation=1, enable_rotation=1, enable_normal_strain=1,
                           enable_shear_strain=1, use_def_gradients=0)
    out = Output(p, fields=["COORDINATE_X", "COORDINATE_Y", "DISPLACEMENT_X", "DISPLACEMENT_Y"], delimiter=",",
                 omit_row_id=True)
    return frames, p, out, [str(GOLD["incremental_gold_text_%d" % k]) for k in range(6)]


def _check_incremental_files(tmp_path, out, rows, golds):
    from test_results import REGRESSION_FLOOR, REGRESSION_TOL
    from dice_b200.results import diff_text
    for k, (r, gold) in enumerate(zip(rows, golds)):
        out.set_images(ref_image="../../component/images/defSyntheticSpeckled%d.tif" % max(k - 1, 0),
                       def_image="../../component/images/defSyntheticSpeckled%d.tif" % k)
        out.write_frame(tmp_path, "DICe_solution", k, r, first_frame=0, num_frames=6, separate_files=False)
        n, rep = diff_text(gold, open(tmp_path / ("DICe_solution_%d.txt" % k)).read(), tol=REGRESSION_TOL,
                           floor=REGRESSION_FLOOR)
        assert n == 0, rep


def test_oracle_incremental_regression(tmp_path):
    frames, p, out, golds = _incremental_regression()
    rows = O.execute_sequence(p, frames[0], frames, syn.init_fields(np.array([42.0]), np.array([42.0])))
    _check_incremental_files(tmp_path, out, rows, golds)


@pytest.mark.gpu
def test_gpu_incremental_regression(tmp_path):
    _need_gpu()
    from dice_b200.schema import Schema
    frames, p, out, golds = _incremental_regression()
    rows = []
    with Schema(p) as s:
        s.set_ref_image(frames[0])
        s.set_fields(syn.init_fields(np.array([42.0]), np.array([42.0])))
        for k, d in enumerate(frames):
            if k > 0:
                s.set_ref_from_def()
            s.set_def_image(d)
            s.execute_correlation()
            rows.append(s.fields())
        assert s.device_status() == 0
    _check_incremental_files(tmp_path, out, rows, golds)
