"""The per-subset Objective entry points of the C ABI on their own:
dicegpu_compute_update_fast (Objective_ZNSSD::computeUpdateFast,
DICe_Objective.cpp:430-657), dicegpu_compute_update_robust
(Objective::computeUpdateRobust, :369-388) and dicegpu_sigma
(Objective::sigma, :150-184), each against the oracle's restatement of the
same entry point on a fresh subset."""
import numpy as np
import pytest

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O
from tests._exact import assert_rows_equal


def _case(shape=abi.AFFINE_SF, w=192, h=160, step=14):
    ref, deff = syn.config1(w=w, h=h)
    ref, deff = ref.numpy(), deff.numpy()
    cx, cy = syn.grid_points(w, h, 21, step)
    kw = dict(subset_size=21, fast_solver_tolerance=1e-5)
    if shape == abi.AFFINE_SF:
        kw.update(enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1)
    else:
        kw.update(shape_function=abi.QUADRATIC_SF, fast_solver_tolerance=1e-4)
    p = abi.default_params(**kw)
    f = syn.init_fields(cx, cy, quadratic=(shape == abi.QUADRATIC_SF))
    return ref, deff, p, f


def test_oracle_objective_entries_agree_with_the_frame():
    """The oracle's Gauss-Newton entry gives the same parameters as the full
    correlation routine on the first frame (same initial guess)."""
    ref, deff, p, f = _case()
    g = f.copy()
    it, st = O.objective(p, ref, deff, g, 0)
    fr = f.copy()
    O.execute_frame(p, ref, deff, fr, first_frame=True, nthreads=4)
    ok = (st == abi.CORRELATION_SUCCESSFUL) & (fr[:, abi.F_STATUS] < 2)
    assert ok.mean() > 0.9
    assert np.array_equal(g[ok, abi.F_DISP_X], fr[ok, abi.F_DISP_X])
    assert np.array_equal(it[ok], fr[ok, abi.F_ITERATIONS].astype(np.int32))


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _schema(p, ref, deff, f):
    from dice_b200.schema import Schema
    s = Schema(p)
    s.set_ref_image(ref)
    s.set_fields(f)
    s.set_def_image(deff)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [abi.AFFINE_SF, abi.QUADRATIC_SF])
def test_compute_update_fast_matches_oracle(shape):
    _gpu()
    ref, deff, p, f = _case(shape)
    with _schema(p, ref, deff, f) as s:
        g, it, st = s.compute_update_fast(f)
    o = f.copy()
    oit, ost = O.objective(p, ref, deff, o, 0)
    assert np.array_equal(st, ost)
    ok = ost == abi.CORRELATION_SUCCESSFUL
    assert ok.mean() > 0.9
    assert np.array_equal(it, oit)
    assert_rows_equal(g, o, cols=[abi.F_DISP_X + i for i in range(6)] + [abi.F_QUAD_A + i for i in range(12)] +
                      [abi.F_CONDITION])
    # the true motion of the synthetic pair
    assert np.median(np.abs(g[ok, abi.F_DISP_X] - 0.37)) < 0.02


@pytest.mark.gpu
def test_compute_update_robust_matches_oracle():
    _gpu()
    ref, deff, p, f = _case()
    p = abi.default_params(subset_size=21, enable_rotation=1)
    with _schema(p, ref, deff, f) as s:
        g, it, st = s.compute_update_robust(f)
    o = f.copy()
    oit, ost = O.objective(p, ref, deff, o, 1)
    assert np.array_equal(st, ost)
    ok = ost == abi.CORRELATION_SUCCESSFUL
    assert ok.mean() > 0.9
    assert np.array_equal(it, oit)
    assert_rows_equal(g, o, cols=[abi.F_DISP_X + i for i in range(6)])


@pytest.mark.gpu
@pytest.mark.parametrize("defgrad", [0, 1])
def test_sigma_matches_oracle(defgrad):
    _gpu()
    ref, deff, p, f = _case()
    p.use_def_gradients = defgrad
    f = f.copy()
    f[:, abi.F_DISP_X] = 0.37
    f[:, abi.F_DISP_Y] = -1.21
    with _schema(p, ref, deff, f) as s:
        sg, no = s.sigma(f)
    osg, ono = O.objective(p, ref, deff, f.copy(), 2)
    assert np.all(sg > 0)
    assert np.array_equal(sg, osg)
    assert np.array_equal(no, ono)


@pytest.mark.gpu
@pytest.mark.parametrize("optimization", [abi.GRADIENT_BASED, abi.SIMPLEX])
def test_beta_output_matches_oracle(optimization):
    """Objective::beta (DICe_Objective.cpp:78-148), written to the BETA
    column when params.output_beta is set: on every converged subset of a
    frame, equal to the oracle's, and present (non-zero somewhere)."""
    _gpu()
    from dice_b200.schema import Schema
    ref, deff, p, f = _case()
    p.output_beta = 1
    p.optimization = optimization
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_fields(f)
        s.set_def_image(deff)
        s.execute_correlation()
        g = s.fields()
    o = f.copy()
    O.execute_frame(p, ref, deff, o, first_frame=True, nthreads=4)
    assert_rows_equal(g, o)
    ok = o[:, abi.F_STATUS] < 2
    assert ok.mean() > 0.9
    assert np.all(np.isfinite(g[ok, abi.F_BETA]))
    assert np.any(g[ok, abi.F_BETA] != 0)
