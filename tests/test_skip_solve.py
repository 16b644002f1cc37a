"""Skipped solves (SKIP_SOLVE in a subset file, params.skip_all_solves;
Schema::generic_correlation_routine, DICe_Schema.cpp:2051-2059, 2118-2143).

A skipped subset is initialised from its field values, evaluated there --
sigma, gamma, beta, contrast, active pixels -- and recorded with
STATUS_FLAG = FRAME_SKIPPED and ITERATIONS = -1, without the optimiser or
the jump and gamma tests.  The oracle restates that branch; the GPU equals
the oracle bit for bit over a two-frame sequence with per-subset flags that
change between the frames, and with every solve skipped."""
import numpy as np
import pytest

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O
from tests._exact import assert_rows_equal


def _case():
    ref, deff = syn.config1(w=192, h=160)
    ref, deff = ref.numpy(), deff.numpy()
    cx, cy = syn.grid_points(192, 160, 21, 14)
    f = syn.init_fields(cx, cy)
    f[:, abi.F_DISP_X] = 0.2
    return ref, deff, f


def _params(**kw):
    base = dict(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                fast_solver_tolerance=1e-5)
    base.update(kw)
    return abi.default_params(**base)


def test_oracle_skipped_subsets_keep_their_guess():
    ref, deff, f = _case()
    p = _params()
    skip = np.zeros(len(f), np.uint8)
    skip[::3] = 1
    o = f.copy()
    O.execute_frame(p, ref, deff, o, first_frame=True, nthreads=4, skip_solve=skip)
    s = skip == 1
    assert (o[s, abi.F_STATUS] == abi.FRAME_SKIPPED).all() and (o[s, abi.F_ITERATIONS] == -1).all()
    assert (o[s, abi.F_DISP_X] == np.float32(0.2)).all()
    assert (o[s, abi.F_GAMMA] > 0).all() and (o[s, abi.F_SIGMA] > 0).all()
    assert (o[~s, abi.F_STATUS] < 2).mean() > 0.9
    pa = _params(skip_all_solves=1)
    oa = f.copy()
    O.execute_frame(pa, ref, deff, oa, first_frame=True, nthreads=4)
    assert (oa[:, abi.F_STATUS] == abi.FRAME_SKIPPED).all()
    assert np.array_equal(oa[s], o[s])


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


@pytest.mark.gpu
@pytest.mark.parametrize("beta", [0, 1])
def test_gpu_skip_solve_matches_oracle(beta):
    _gpu()
    from dice_b200.schema import Schema
    ref, deff, f = _case()
    ref2 = np.ascontiguousarray(np.roll(deff, 1, axis=1))   # a second frame one pixel further along x
    p = _params(output_beta=beta)
    rng = np.random.default_rng(7)
    flags = [(rng.random(len(f)) < 0.3).astype(np.uint8), (rng.random(len(f)) < 0.3).astype(np.uint8)]
    o = f.copy()
    want = []
    for k, fl in enumerate(flags):
        O.execute_frame(p, ref, ref2 if k else deff, o, first_frame=(k == 0), nthreads=4, skip_solve=fl)
        want.append(o.copy())
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        got = []
        for k, fl in enumerate(flags):
            s.set_skip_solve(fl)
            s.set_def_image(ref2 if k else deff)
            s.execute_correlation()
            got.append(s.fields())
        assert s.device_status() == 0
    for g, w in zip(got, want):
        assert_rows_equal(g, w)
    assert (got[0][flags[0] == 1, abi.F_STATUS] == abi.FRAME_SKIPPED).all()


@pytest.mark.gpu
def test_gpu_skip_all_solves_matches_oracle():
    _gpu()
    from dice_b200.schema import Schema
    ref, deff, f = _case()
    p = _params(skip_all_solves=1)
    o = f.copy()
    O.execute_frame(p, ref, deff, o, first_frame=True, nthreads=4)
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        s.set_def_image(deff)
        s.execute_correlation()
        g = s.fields()
    assert_rows_equal(g, o)
    assert (g[:, abi.F_STATUS] == abi.FRAME_SKIPPED).all()
