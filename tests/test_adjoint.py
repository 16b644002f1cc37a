"""Adjoint of the subset objective (dicegpu_adjoint, the libtorch autograd
Function over it, and the B-spline fit that uses it).

Checks:
* the objective values equal Objective::gamma (dicegpu_gamma / the oracle);
* d/dparams and d/d(deformed intensities) against central finite
  differences of an FP64 evaluation of the same forward map (h = 1e-3 px,
  scaled by the subset half-width for the dimensionless parameters; 0.01
  grey levels for the image), to 1e-5 relative;
* the least-squares objective's derivative through the interpolated
  gradient images against twice the Gauss-Newton right-hand side q that the
  oracle assembles (DICe_Objective.cpp:523-546);
* the autograd Function returns the same gradients as the direct call;
* a 16 x 16 B-spline control grid fitted by gradient descent through the
  adjoint recovers the imposed field and agrees with per-subset Gauss-Newton.
"""
import numpy as np
import pytest
import torch

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O


# ---------------------------------------------------------------------------
# FP64 forward map (test checker): affine / quadratic warp, Keys fourth-order
# interpolation, gamma or the least-squares objective over active pixels.
# ---------------------------------------------------------------------------
def _keys(s):
    s = np.abs(s)
    return np.where(s < 1.0, 4.0 / 3.0 * s ** 3 - 7.0 / 3.0 * s ** 2 + 1.0,
                    np.where(s < 2.0, -7.0 / 12.0 * s ** 3 + 3.0 * s ** 2 - 59.0 / 12.0 * s + 2.5,
                             np.where(s < 3.0, 1.0 / 12.0 * s ** 3 - 2.0 / 3.0 * s ** 2 + 1.75 * s - 1.5, 0.0)))


def _round_pixel(m):
    i = np.trunc(m)
    return np.where(np.trunc(m + 0.5) == i, i, i + 1).astype(np.int64)


def forward64(ref, deff, cx, cy, half, P, quadratic=False, objective=0):
    """Objective per subset; P is (n, 6) affine (u, v, theta, ex, ey, gxy) or
    (n, 12) quadratic, all float64."""
    h, w = deff.shape
    d = np.arange(-half, half + 1, dtype=np.float64)
    dy, dx = np.meshgrid(d, d, indexing="ij")
    dx, dy = dx.ravel()[None, :], dy.ravel()[None, :]
    cxa, cya = np.asarray(cx, np.float64)[:, None], np.asarray(cy, np.float64)[:, None]
    if quadratic:
        A = [P[:, k][:, None] for k in range(12)]
        mx = A[0] * dx + A[1] * dy + A[2] * dx * dy + A[3] * dx * dx + A[4] * dy * dy + A[5] + cxa
        my = A[6] * dx + A[7] * dy + A[8] * dx * dy + A[9] * dx * dx + A[10] * dy * dy + A[11] + cya
    else:
        u, v, t, ex, ey, g = [P[:, k][:, None] for k in range(6)]
        Dx = (1.0 + ex) * dx + g * dy
        Dy = (1.0 + ey) * dy + g * dx
        mx = np.cos(t) * Dx - np.sin(t) * Dy + u + cxa
        my = np.sin(t) * Dx + np.cos(t) * Dy + v + cya
    px, py = _round_pixel(mx), _round_pixel(my)
    act = (px >= 4) & (px < w - 4) & (py >= 4) & (py < h - 4)
    ix, iy = np.floor(mx).astype(np.int64), np.floor(my).astype(np.int64)
    tx, ty = mx - ix, my - iy
    G = np.zeros_like(mx)
    for m in range(6):
        wy = _keys(ty - (m - 2))
        row = np.clip(iy - 2 + m, 0, h - 1)
        for q in range(6):
            wx = _keys(tx - (q - 2))
            col = np.clip(ix - 2 + q, 0, w - 1)
            G += wy * wx * deff[row, col]
    xs = (cxa + dx).astype(np.int64)
    ys = (cya + dy).astype(np.int64)
    F = ref[ys, xs].astype(np.float64)
    out = np.zeros(P.shape[0])
    for i in range(P.shape[0]):
        a = act[i]
        Gi, Fi = G[i, a], F[i, a]
        Gt, Ft = Gi - Gi.mean(), Fi - Fi.mean()
        if objective == 0:
            out[i] = 2.0 - 2.0 * (Gt * Ft).sum() / np.sqrt((Gt * Gt).sum() * (Ft * Ft).sum())
        else:
            out[i] = ((Gt - Ft) ** 2).sum()
    return out


def _small_case(w=128, h=112, half=10, step=18):
    ref, deff = syn.config1(w=w, h=h)
    ref, deff = ref.numpy(), deff.numpy()
    cx, cy = syn.grid_points(w, h, 2 * half + 1, step)
    keep = (cx >= 24) & (cx <= w - 25) & (cy >= 24) & (cy <= h - 25)
    return ref, deff, cx[keep], cy[keep]


def test_forward64_matches_oracle_gamma():
    ref, deff, cx, cy = _small_case()
    p = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1)
    f = syn.init_fields(cx, cy)
    rng = np.random.default_rng(0)
    P = np.zeros((len(cx), 6))
    P[:, 0] = 0.37 + rng.normal(0, 0.2, len(cx))
    P[:, 1] = -1.21 + rng.normal(0, 0.2, len(cx))
    P[:, 2] = rng.normal(0, 0.01, len(cx))
    P[:, 3:] = rng.normal(0, 0.005, (len(cx), 3))
    f[:, abi.F_DISP_X:abi.F_DISP_X + 6] = P
    g_or = O.gamma(p, ref, deff, f)
    g64 = forward64(ref, deff.astype(np.float64), cx, cy, 10, P.astype(np.float32).astype(np.float64))
    assert np.allclose(g64, g_or, rtol=2e-3, atol=2e-5)


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _gpu():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _schema(p, ref, deff, cx, cy):
    from dice_b200.schema import Schema
    s = Schema(p)
    s.set_ref_image(ref)
    s.set_subsets(cx, cy)
    s.set_def_image(deff)
    return s


def _rows(cx, cy, P, quadratic=False):
    f = syn.init_fields(cx, cy, quadratic=quadratic)
    col = abi.F_QUAD_A if quadratic else abi.F_DISP_X
    f[:, col:col + P.shape[1]] = P
    return f


def _fd_params(ref, deff, cx, cy, P, quadratic, objective, half=10, h=1e-3):
    scale = np.ones(P.shape[1])
    if quadratic:
        # A..L: coefficients of dx, dy, dxdy, dx^2, dy^2, 1
        per = np.array([half, half, half * half, half * half, half * half, 1.0])
        scale = 1.0 / np.concatenate([per, per])
    else:
        scale[2:] = 1.0 / half
    out = np.zeros_like(P)
    d64 = deff.astype(np.float64)
    for j in range(P.shape[1]):
        e = np.zeros(P.shape[1])
        e[j] = h * scale[j]
        out[:, j] = (forward64(ref, d64, cx, cy, half, P + e, quadratic, objective) -
                     forward64(ref, d64, cx, cy, half, P - e, quadratic, objective)) / (2 * h * scale[j])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("quadratic", [False, True])
@pytest.mark.parametrize("objective", [0, 1])
def test_adjoint_params_match_finite_differences(quadratic, objective):
    _gpu()
    ref, deff, cx, cy = _small_case()
    rng = np.random.default_rng(1)
    n = len(cx)
    if quadratic:
        p = abi.default_params(subset_size=21, shape_function=abi.QUADRATIC_SF)
        P = np.zeros((n, 12))
        P[:, 0] = P[:, 7] = 1.0
        P[:, 5] = 0.2 + rng.normal(0, 0.1, n)
        P[:, 11] = -0.9 + rng.normal(0, 0.1, n)
        P[:, [1, 6]] = rng.normal(0, 0.004, (n, 2))
        P[:, [2, 3, 4, 8, 9, 10]] = rng.normal(0, 2e-4, (n, 6))
    else:
        p = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1)
        P = np.zeros((n, 6))
        P[:, 0] = 0.2 + rng.normal(0, 0.1, n)
        P[:, 1] = -0.9 + rng.normal(0, 0.1, n)
        P[:, 2] = rng.normal(0, 0.01, n)
        P[:, 3:] = rng.normal(0, 0.005, (n, 3))
    P = P.astype(np.float32).astype(np.float64)   # the parameters the device sees
    with _schema(p, ref, deff, cx, cy) as s:
        rows = torch.from_numpy(_rows(cx, cy, P, quadratic)).cuda()
        val, dp = s.adjoint(rows, objective=objective)
        val, dp = val.cpu().numpy(), dp.cpu().numpy()[:, :P.shape[1]]
    fd = _fd_params(ref, deff, cx, cy, P, quadratic, objective)
    v64 = forward64(ref, deff.astype(np.float64), cx, cy, 10, P, quadratic, objective)
    assert np.allclose(val, v64, rtol=1e-4, atol=1e-6)
    # relative error per parameter, |d - fd| over the largest |fd| of the
    # column: at most 1e-5 (measured 0.9e-6 .. 9.8e-6 on these cases; h = 1e-4
    # gives the same figures, so they are the FP32 evaluation's rounding,
    # not the differences' truncation)
    for j in range(P.shape[1]):
        rel = np.max(np.abs(dp[:, j] - fd[:, j])) / np.abs(fd[:, j]).max()
        assert rel <= 1e-5, (j, rel, dp[:4, j], fd[:4, j])


@pytest.mark.gpu
def test_adjoint_values_equal_gamma_entry():
    _gpu()
    ref, deff, cx, cy = _small_case()
    p = abi.default_params(subset_size=21, enable_rotation=1)
    P = np.zeros((len(cx), 6))
    P[:, 0], P[:, 1] = 0.3, -1.1
    f = _rows(cx, cy, P)
    with _schema(p, ref, deff, cx, cy) as s:
        g = s.gamma(f)
        val, _ = s.adjoint(torch.from_numpy(f).cuda())
    assert np.allclose(val.cpu().numpy(), g, rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
def test_adjoint_image_derivative_matches_finite_differences():
    _gpu()
    ref, deff, cx, cy = _small_case()
    p = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1)
    n = len(cx)
    rng = np.random.default_rng(2)
    P = np.zeros((n, 6))
    P[:, 0] = 0.25 + rng.normal(0, 0.1, n)
    P[:, 1] = -1.0 + rng.normal(0, 0.1, n)
    P = P.astype(np.float32).astype(np.float64)
    seed = rng.uniform(0.5, 1.5, n)
    with _schema(p, ref, deff, cx, cy) as s:
        ddef = torch.zeros(deff.shape, dtype=torch.float32, device="cuda")
        s.adjoint(torch.from_numpy(_rows(cx, cy, P)).cuda(), seed=torch.from_numpy(seed).cuda(), ddef=ddef)
        ddef = ddef.cpu().numpy().astype(np.float64)
    d64 = deff.astype(np.float64)
    loss = lambda img: float((seed * forward64(ref, img, cx, cy, 10, P)).sum())  # noqa: E731
    # pixels inside subsets (several subsets overlap near the centre), and one outside all of them
    picks = [(int(cy[0]), int(cx[0])), (int(cy[0]) + 3, int(cx[0]) - 5), (int(cy[-1]) - 2, int(cx[-1]) + 4),
             (int(cy[len(cy) // 2]), int(cx[len(cx) // 2]) + 9), (2, 2)]
    hstep = 0.01
    scale = np.abs(ddef).max()
    for (y, x) in picks:
        a, b = d64.copy(), d64.copy()
        a[y, x] += hstep
        b[y, x] -= hstep
        fd = (loss(a) - loss(b)) / (2 * hstep)
        # relative to the largest derivative over the image, at most 1e-5
        assert abs(ddef[y, x] - fd) <= 1e-5 * scale, (y, x, ddef[y, x], fd, abs(ddef[y, x] - fd) / scale)
    assert ddef[2, 2] == 0.0


@pytest.mark.gpu
def test_least_squares_adjoint_is_twice_gauss_newton_rhs():
    _gpu()
    ref, deff, cx, cy = _small_case()
    p = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           use_def_gradients=1)
    n = len(cx)
    rng = np.random.default_rng(3)
    P = np.zeros((n, 6))
    P[:, 0] = 0.3 + rng.normal(0, 0.1, n)
    P[:, 1] = -1.1 + rng.normal(0, 0.1, n)
    P[:, 2:] = rng.normal(0, 0.003, (n, 4))
    f = _rows(cx, cy, P)
    _, q = O.gn_system(p, ref, deff, f, 6)
    with _schema(p, ref, deff, cx, cy) as s:
        _, dp = s.adjoint(torch.from_numpy(f).cuda(), objective=1, grad_source=1)
        dp = dp.cpu().numpy()[:, :6]
    for j in range(6):
        tol = 1e-4 * np.abs(q[:, j]).max()
        assert np.max(np.abs(dp[:, j] - 2.0 * q[:, j])) < 2 * tol, j


@pytest.mark.gpu
def test_autograd_function_gradients():
    _gpu()
    from dice_b200 import autograd
    ref, deff, cx, cy = _small_case()
    p = abi.default_params(subset_size=21, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1)
    n = len(cx)
    rng = np.random.default_rng(4)
    P = np.zeros((n, 6))
    P[:, 0] = 0.3 + rng.normal(0, 0.1, n)
    P[:, 1] = -1.0 + rng.normal(0, 0.1, n)
    with _schema(p, ref, deff, cx, cy) as s:
        params = torch.from_numpy(P).cuda().requires_grad_(True)
        img = torch.from_numpy(deff).cuda().requires_grad_(True)
        w = torch.from_numpy(rng.uniform(0.5, 1.5, n)).cuda()
        val = autograd.subset_objective(params, img, s)
        (val * w).sum().backward()
        ddef = torch.zeros_like(img)
        v2, dp2 = s.adjoint(torch.from_numpy(_rows(cx, cy, P)).cuda(), seed=w.contiguous(), ddef=ddef)
        assert torch.allclose(val.detach(), v2)
        assert torch.allclose(params.grad, dp2[:, :6], rtol=1e-6, atol=1e-9)
        assert torch.allclose(img.grad, ddef, rtol=1e-5, atol=1e-7)


@pytest.mark.gpu
def test_bspline_fit_recovers_field_and_agrees_with_gauss_newton():
    _gpu()
    from dice_b200 import bspline
    from dice_b200.schema import Schema
    w = h = 512
    ref, deff, field, ctrl = syn.config4(device="cuda", w=w, h=h, ncontrol=10)
    cx, cy = syn.grid_points(w, h, 25, 14)
    p = abi.default_params(subset_size=25, enable_rotation=1, enable_normal_strain=1, enable_shear_strain=1,
                           fast_solver_tolerance=1e-5)
    with Schema(p) as s:
        s.set_ref_image(ref)
        s.set_subsets(cx, cy)
        s.set_def_image(deff)
        s.execute_correlation()
        gn = s.fields()
        tcx = torch.from_numpy(cx).cuda()
        tcy = torch.from_numpy(cy).cuda()
        fit = bspline.fit(s, deff, field, tcx, tcy, iters=300, lr=0.05)
    ut, vt = field.eval(ctrl, tcx, tcy)
    uf, vf = field.eval(fit, tcx, tcy)
    ok = torch.from_numpy(gn[:, abi.F_STATUS] < 2).cuda()
    ug = torch.from_numpy(gn[:, abi.F_DISP_X]).cuda()
    vg = torch.from_numpy(gn[:, abi.F_DISP_Y]).cuda()
    err_fit = bspline.rms(torch.cat([(uf - ut)[ok], (vf - vt)[ok]]))
    err_gn = bspline.rms(torch.cat([(ug - ut)[ok], (vg - vt)[ok]]))
    gap = bspline.rms(torch.cat([(uf - ug)[ok], (vf - vg)[ok]]))
    assert ok.float().mean() > 0.95
    assert err_gn < 0.05
    assert err_fit < 0.05
    assert gap < 0.06
