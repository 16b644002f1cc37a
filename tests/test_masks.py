"""Obstructions and blocking subsets on the GPU, against the oracle and the
reference's regression gold.

* conformal_subset_def and simple_obstruction run end to end on the device
  (subset file -> shapes -> correlation -> result files) and pass the
  reference's own regression comparison (DICe_Diff -t 0.05 -f 5.0E-5).
* examples/obstruction runs with subset evolution (tracking defaults): the
  device's per-pixel evolution state and turned-on reference intensities
  equal the oracle's frame by frame, and the example's gold passes its own
  comparison (DICe_Diff -t 10.0 -f 1E-4).
* Random conformal subsets with obstructed regions and blocking lists run
  under the tracking routine on the device and in the oracle: status flags
  and active-pixel counts (the masks' effect) are equal, the Gauss-Newton
  results agree within 1e-4 px.
"""
import numpy as np
import pytest
import torch

from dice_b200 import abi
from dice_b200 import synthetic as syn
from dice_b200.results import diff_text
from dice_b200.schema import Schema
from oracle import oracle as O
from tests._exact import assert_rows_equal
from test_results import (GOLD, REGRESSION_FLOOR, REGRESSION_TOL, blocking_csr, check_example_files,
                          conformal_subset_def_case, obstruction_example_case, oracle_obstruction_example,
                          simple_obstruction_case)

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _gold_check(tmp_path, out, rows_per_frame, gold_texts):
    for k, f in enumerate(rows_per_frame):
        out.write_frame(tmp_path, "DICe_solution", k, f)
    for i, text in enumerate(gold_texts):
        n, rep = diff_text(text, open(tmp_path / ("DICe_solution_%d.txt" % i)).read(), tol=REGRESSION_TOL,
                           floor=REGRESSION_FLOOR)
        assert n == 0, rep


def test_gpu_conformal_subset_def_gold(tmp_path):
    _need_gpu()
    sf, p, ref, deff, out = conformal_subset_def_case()
    with Schema(p) as s:
        s.set_ref_image(ref)
        sf.apply(s)
        s.set_def_image(deff)
        s.execute_correlation()
        g = s.fields()
        assert s.device_status() == 0
    _gold_check(tmp_path, out, [g], [str(GOLD["conformal_subset_def_gold_text_%d" % k]) for k in range(5)])
    o = syn.init_fields(sf.coordinates[:, 0], sf.coordinates[:, 1])
    offs, ids = blocking_csr(sf)
    O.execute_frame_shapes(p, ref, deff, o, sf.shapes, sf.vx, sf.vy, offs, ids, force_simplex=sf.force_simplex)
    assert_rows_equal(g, o)


def test_gpu_simple_obstruction_gold(tmp_path):
    _need_gpu()
    sf, p, frames, out = simple_obstruction_case()
    rows = []
    o = syn.init_fields(sf.coordinates[:, 0], sf.coordinates[:, 1])
    ref = frames[0]
    with Schema(p) as s:
        s.set_ref_image(ref)
        sf.apply(s)
        for k in range(frames.shape[0]):
            s.set_def_image(frames[k])
            s.execute_correlation()
            g = s.fields()
            rows.append(g)
            O.execute_frame_shapes(p, ref.astype(np.float32), frames[k].astype(np.float32), o, sf.shapes, sf.vx,
                                   sf.vy, first_frame=(k == 0))
            assert g[0, abi.F_STATUS] == o[0, abi.F_STATUS]
            assert g[0, abi.F_ACTIVE_PIXELS] == o[0, abi.F_ACTIVE_PIXELS], k
            assert abs(g[0, abi.F_DISP_X] - o[0, abi.F_DISP_X]) < 5e-3
        assert s.device_status() == 0
    _gold_check(tmp_path, out, rows, [str(GOLD["simple_obstruction_gold_text"])])


def _blocking_case(seed, n_side=5):
    """A grid of conformal subsets (polygons and rectangles), some with an
    obstructed region, each blocked by one or two neighbours (earlier and
    later in index order) on a translated speckle pair."""
    rng = np.random.default_rng(seed)
    w = h = 320
    ref_t = syn.speckle_image(w, h, seed=seed, r_min=2, r_max=4, grey_lo=20, grey_hi=230, blur_sigma=0.8)
    shift = (1.3, -0.7)
    deff = syn.warp_image(ref_t, lambda X, Y: (torch.full_like(X, shift[0]), torch.full_like(Y, shift[1])),
                          noise_sigma=1.0, seed=seed + 50, clip=(0, 255)).numpy()
    ref = ref_t.numpy()
    shapes, vx, vy, cx, cy, blockers = [], [], [], [], [], []
    step = (w - 80) // (n_side - 1)
    for j in range(n_side):
        for i in range(n_side):
            k = len(cx)
            x, y = 40 + i * step, 40 + j * step
            cx.append(x)
            cy.append(y)
            if rng.random() < 0.5:
                shapes.append(abi.rectangle(k, x, y, int(rng.integers(21, 35)), int(rng.integers(21, 35))))
            else:
                m = int(rng.integers(4, 8))
                ang = np.sort(rng.uniform(0, 2 * np.pi, m))
                rad = rng.uniform(12, 20, m)
                shapes.append(abi.polygon(k, len(vx), m))
                vx += list(np.round(x + rad * np.cos(ang)).astype(int))
                vy += list(np.round(y + rad * np.sin(ang)).astype(int))
            if rng.random() < 0.4:
                shapes.append(abi.rectangle(k, x + int(rng.integers(-12, 13)), y + int(rng.integers(-12, 13)),
                                            int(rng.integers(6, 16)), int(rng.integers(6, 16)),
                                            role=abi.ROLE_OBSTRUCTED))
    n = len(cx)
    for k in range(n):
        nb = [k - 1, k + 1, k - n_side, k + n_side]
        nb = [b for b in nb if 0 <= b < n]
        pick = list(rng.choice(nb, size=int(rng.integers(0, 3)), replace=False))
        blockers.append(sorted(int(b) for b in pick))
    return ref, deff, np.asarray(cx, float), np.asarray(cy, float), shapes, np.asarray(vx, np.int32), \
        np.asarray(vy, np.int32), blockers


@pytest.mark.parametrize("seed, skin", [(11, 1.0), (12, 1.3)])
def test_gpu_blocking_tracking_matches_oracle(seed, skin):
    """Tracking routine with blocking, Gauss-Newton kept on (override), two
    frames so that blocked masks see both this frame's and the snapshot's
    parameters."""
    _need_gpu()
    ref, deff, cx, cy, shapes, vx, vy, blockers = _blocking_case(seed)
    p = abi.default_params(subset_size=0, enable_rotation=1, correlation_routine=abi.TRACKING_ROUTINE,
                           override_force_simplex=1, obstruction_skin_factor=skin, fast_solver_tolerance=1e-5)
    f0 = syn.init_fields(cx, cy)
    f0[:, abi.F_DISP_X] = 1.0
    offs = np.zeros(len(cx) + 1, np.int32)
    ids = []
    for i, b in enumerate(blockers):
        ids += b
        offs[i + 1] = offs[i] + len(b)
    ids = np.asarray(ids, np.int32)
    frames = [deff, deff]
    gs = []
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f0)
        s.set_subset_shapes(shapes, vx, vy)
        s.set_blocking(blockers)
        for d in frames:
            s.set_def_image(d)
            s.execute_correlation()
            gs.append(s.fields())
        assert s.device_status() == 0
    o = f0.copy()
    for k, d in enumerate(frames):
        O.execute_frame_shapes(p, ref, d, o, shapes, vx, vy, offs, ids, first_frame=(k == 0))
        g = gs[k]
        assert_rows_equal(g, o)
        assert (o[:, abi.F_STATUS] < 2).mean() > 0.8
    # blocking and obstruction deactivated pixels somewhere
    full = np.asarray(O.rasterize(len(cx), [sh for sh in shapes if sh.role == 0], vx, vy)[0])
    npix = np.diff(full)
    assert (gs[-1][:, abi.F_ACTIVE_PIXELS] < npix).sum() >= 3


def test_gpu_generic_routine_forces_simplex_on_blocking():
    """Generic routine: no blocked masks, but blocked and blocking subsets
    take the simplex unless override_force_simplex."""
    _need_gpu()
    ref, deff, cx, cy, shapes, vx, vy, blockers = _blocking_case(13, n_side=4)
    p = abi.default_params(subset_size=0, correlation_routine=abi.GENERIC_ROUTINE)
    f0 = syn.init_fields(cx, cy)
    f0[:, abi.F_DISP_X] = 1.0
    offs = np.zeros(len(cx) + 1, np.int32)
    ids = []
    for i, b in enumerate(blockers):
        ids += b
        offs[i + 1] = offs[i] + len(b)
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f0)
        s.set_subset_shapes(shapes, vx, vy)
        s.set_blocking(blockers)
        s.set_def_image(deff)
        s.execute_correlation()
        g = s.fields()
    o = f0.copy()
    O.execute_frame_shapes(p, ref, deff, o, shapes, vx, vy, offs, np.asarray(ids, np.int32))
    assert np.array_equal(g[:, abi.F_STATUS], o[:, abi.F_STATUS])
    assert np.array_equal(g[:, abi.F_ACTIVE_PIXELS], o[:, abi.F_ACTIVE_PIXELS])
    involved = np.zeros(len(cx), bool)
    for i, b in enumerate(blockers):
        if b:
            involved[i] = True
            involved[b] = True
    # simplex iterations run to tens; Gauss-Newton stops within a handful
    assert np.median(g[involved, abi.F_ITERATIONS]) > np.median(g[~involved, abi.F_ITERATIONS])
    ok = o[:, abi.F_STATUS] < 2
    assert np.max(np.abs(g[ok, abi.F_DISP_X] - o[ok, abi.F_DISP_X])) < 5e-3


def test_gpu_blocking_rejects_circle_blockers_and_plain_path():
    _need_gpu()
    p = abi.default_params(subset_size=0, correlation_routine=abi.TRACKING_ROUTINE)
    ref = np.zeros((64, 64), np.float32)
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_subsets(np.array([20.0, 40.0]), np.array([20.0, 40.0]))
        s.set_subset_shapes([abi.circle(0, 20, 20, 5.0), abi.rectangle(1, 40, 40, 9, 9)])
        with pytest.raises(RuntimeError) as e:
            s.set_blocking([[1], [0]])          # subset 0's circle boundary cannot be deformed
        assert "UNSUPPORTED" in str(e.value)
        s.set_blocking([[], [1]])               # a rectangle blocker is fine
        s.set_def_image(ref)
        with pytest.raises(RuntimeError):
            abi.check(s.lib.dicegpu_execute_correlation_plain(s.ctx), "plain")
        s.set_blocking(None)


def test_gpu_blocking_sequence_graph_equals_frame_calls():
    """A frame sequence captured as one CUDA graph (tracking waves, blocked
    bitmaps rebuilt per frame inside it) gives the fields of frame-by-frame
    calls bit for bit."""
    _need_gpu()
    ref, deff, cx, cy, shapes, vx, vy, blockers = _blocking_case(14, n_side=4)
    deff2 = syn.warp_image(torch.from_numpy(ref), lambda X, Y: (torch.full_like(X, 1.6), torch.full_like(Y, -0.4)),
                           noise_sigma=1.0, seed=77, clip=(0, 255)).numpy()
    frames = [deff, deff2, deff]
    p = abi.default_params(subset_size=0, enable_rotation=1, correlation_routine=abi.TRACKING_ROUTINE,
                           override_force_simplex=1, obstruction_skin_factor=1.2)
    f0 = syn.init_fields(cx, cy)
    f0[:, abi.F_DISP_X] = 1.0

    def setup(s):
        s.set_ref_image(ref)
        s.set_fields(f0)
        s.set_subset_shapes(shapes, vx, vy)
        s.set_blocking(blockers)

    with Schema(p) as s:
        setup(s)
        for d in frames:
            s.set_def_image(d)
            s.execute_correlation()
        want = s.fields()
    with Schema(p) as s:
        setup(s)
        s.capture_sequence([torch.from_numpy(d).cuda() for d in frames],
                           reset_fields=torch.from_numpy(f0).cuda())
        s.launch_sequence()
        torch.cuda.synchronize()
        got = s.fields()
        assert s.device_status() == 0
    assert np.array_equal(got, want)


def _device_example(p, sf, frames, graph_check=False):
    rows, states = [], []
    with Schema(p) as s:
        s.set_ref_image(frames[0])
        sf.apply(s)
        f0 = s.fields()
        for k in range(1, len(frames)):
            s.set_def_image(frames[k])
            s.execute_correlation()
            rows.append(s.fields())
            states.append(s.subset_pixel_state())
        assert s.device_status() == 0
        if graph_check:
            # the same sequence as one CUDA graph: the evolution state
            # restarts at its first frame and ends where the frame calls left it
            s.capture_sequence([torch.from_numpy(np.ascontiguousarray(d)).cuda() for d in frames[1:]],
                               reset_fields=torch.from_numpy(f0).cuda())
            s.launch_sequence()
            torch.cuda.synchronize()
            assert np.array_equal(s.fields(), rows[-1])
            g_state, g_vals = s.subset_pixel_state()
            assert np.array_equal(g_state, states[-1][0]) and np.array_equal(g_vals, states[-1][1])
            assert s.device_status() == 0
    return rows, states


def test_gpu_obstruction_example_subset_evolution(tmp_path):
    """The example's own parameters (the blocked subset runs the simplex):
    device and oracle agree in every result column, the evolution state and
    the turned-on reference intensities, frame by frame."""
    _need_gpu()
    sf, p, frames, out = obstruction_example_case()
    want_rows, want_states = oracle_obstruction_example(p, sf, frames)
    rows, states = _device_example(p, sf, frames, graph_check=True)
    for k in range(len(rows)):
        assert_rows_equal(rows[k], want_rows[k])
        assert np.array_equal(states[k][0], want_states[k][0]), k
        on = states[k][0] == 2
        assert np.array_equal(states[k][1][on], want_states[k][1][on]), k
    assert (states[-1][0] == 2).sum() >= 5
    # the example's comparison (the simplex end points of the 17 x 17
    # subset's near-zero rotation differ beyond the regression tolerance)
    res = check_example_files(tmp_path, out, rows)
    assert res[0][0] == 0 and res[1][0] == 0, res


def test_gpu_obstruction_example_subset_evolution_gauss_newton():
    """The same sequence with Gauss-Newton for both subsets (tracking
    defaults leave blocked subsets to params.optimization): device and
    oracle agree in every active pixel, the evolution state and the
    turned-on reference intensities."""
    _need_gpu()
    sf, p, frames, _ = obstruction_example_case()
    p.optimization = abi.GRADIENT_BASED
    want_rows, want_states = oracle_obstruction_example(p, sf, frames)
    rows, states = _device_example(p, sf, frames)
    for k in range(len(rows)):
        assert_rows_equal(rows[k], want_rows[k])
        assert np.array_equal(states[k][0], want_states[k][0]), k
        on = states[k][0] == 2
        assert np.array_equal(states[k][1][on], want_states[k][1][on]), k
    assert (states[-1][0] == 2).sum() >= 5
