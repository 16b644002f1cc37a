"""Batched execution: CUDA-graph frame sequences, the launch-shape autotuner
and the persistent work queue, checked against the plain host-driven path
(bit for bit: the same kernels run in the same order on the same data)."""
import numpy as np
import pytest
import torch

from dice_b200 import abi
from dice_b200 import synthetic as syn
from dice_b200.schema import Schema

pytestmark = pytest.mark.gpu


def _setup(w=256, nframes=3):
    dev = torch.device("cuda", 0)
    ref = syn.speckle_image(w, w, seed=2, r_min=3, r_max=5, grey_lo=1000, grey_hi=64000, blur_sigma=0.8,
                            device=dev)
    frames = [syn.warp_image(ref, syn.config2_field(k + 1, nframes), noise_sigma=50.0, seed=200 + k,
                             clip=(0, 65535)) for k in range(nframes)]
    cx, cy = syn.grid_points(w, w, 31, 7)
    p = abi.default_params(subset_size=31, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           fast_solver_tolerance=1e-5)
    return p, ref, frames, cx, cy


def test_graph_sequence_matches_host_loop():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p, ref, frames, cx, cy = _setup()
    f0 = syn.init_fields(cx, cy)
    # host loop
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f0)
        for fr in frames:
            s.set_def_image(fr)
            s.execute_correlation()
        host = s.fields()
    # one graph for the whole sequence, replayed twice from the same start
    stream = torch.cuda.Stream()
    with Schema(p, stream=stream) as g:
        g.set_ref_image(ref)
        g.set_fields(f0)
        reset = torch.from_numpy(f0).cuda()
        torch.cuda.synchronize()
        g.capture_sequence(frames, reset_fields=reset)
        n0 = g.launch_count()
        g.launch_sequence()
        first = g.fields()
        g.launch_sequence()
        second = g.fields()
        assert g.launch_count() - n0 == 2 * 3 * len(frames)   # gradients, pack, frame per frame
    assert np.array_equal(first, host)
    assert np.array_equal(second, host)


def test_autotune_keeps_results():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p, ref, frames, cx, cy = _setup(nframes=1)
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_subsets(cx, cy)
        s.set_def_image(frames[0])
        w, c, ms = s.autotune()
        assert w in (2, 4, 8) and c >= 0 and ms > 0
        assert s.launch_shape() == (w, c)
        s.execute_correlation()
        tuned = s.fields()
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_subsets(cx, cy)
        s.set_def_image(frames[0])
        s.execute_correlation()
        plain = s.fields()
    # the results do not depend on the launch shape
    assert np.array_equal(tuned, plain)


@pytest.mark.parametrize("shape", [(1, 1), (2, 0), (4, 0), (8, 3)])
def test_launch_shapes_give_identical_results(shape):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    p, ref, frames, cx, cy = _setup(nframes=1)
    out = []
    # the default shape first: this small frame runs on eight-warp CTAs
    for sh in [None, shape]:
        with Schema(p) as s:
            if sh is not None:
                s.set_launch_shape(*sh)
            s.set_ref_image(ref)
            s.set_subsets(cx, cy)
            s.set_def_image(frames[0])
            s.execute_correlation()
            out.append(s.fields())
    assert np.array_equal(out[0], out[1])
