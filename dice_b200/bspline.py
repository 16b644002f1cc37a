"""Uniform cubic B-spline displacement fields and their fit through the
subset objective's adjoint.

A field (u, v)(x, y) is a G x G grid of control displacements per component
over the image, spacing s = (extent - 1) / (G - 3), so that the G - 3 spans
cover [0, extent - 1] exactly.  At a point the four basis functions of its
span weigh the 4 x 4 neighbouring control points.

`subset_params` maps the field to per-subset affine shape-function
parameters (u, v, theta, ex, ey, gxy; DICe_LocalShapeFunction.cpp:220-248)
at the subset centres: the deformation gradient F = I + grad(u, v) is split
as F = R(theta) S with S = [[1 + ex, gxy], [gxy, 1 + ey]] symmetric, which is
exactly the affine map's form.  `fit` adjusts the control grid by gradient
descent on the sum of the subsets' gamma, with gradients from the adjoint
kernel (dice_b200.autograd).
"""
import math

import torch


def _basis(t):
    t2 = t * t
    t3 = t2 * t
    return torch.stack([(1.0 - t) ** 3 / 6.0, (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0,
                        (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0, t3 / 6.0], -1)


def _dbasis(t):
    t2 = t * t
    return torch.stack([-0.5 * (1.0 - t) ** 2, 1.5 * t2 - 2.0 * t, -1.5 * t2 + t + 0.5, 0.5 * t2], -1)


class BSplineGrid:
    """Basis of one axis: `dense(coord)` gives the (n x G) weights of the
    control points and their derivative with respect to the coordinate."""

    def __init__(self, extent, ncontrol=16):
        assert ncontrol >= 4
        self.G = ncontrol
        self.spacing = (extent - 1.0) / (ncontrol - 3)

    def dense(self, coord):
        coord = coord.to(torch.float64)
        t = coord / self.spacing
        i = torch.clamp(torch.floor(t), 0, self.G - 4)
        u = t - i
        w = _basis(u)
        dw = _dbasis(u) / self.spacing
        idx = i.long()[:, None] + torch.arange(4, device=coord.device)[None, :]
        W = torch.zeros((coord.numel(), self.G), dtype=torch.float64, device=coord.device)
        dW = torch.zeros_like(W)
        W.scatter_(1, idx, w)
        dW.scatter_(1, idx, dw)
        return W, dW


class BSplineField:
    """Displacement field from a (2, G, G) control tensor (component, row y,
    column x) on a width x height image."""

    def __init__(self, width, height, ncontrol=16):
        self.gx = BSplineGrid(width, ncontrol)
        self.gy = BSplineGrid(height, ncontrol)
        self.G = ncontrol

    def eval(self, ctrl, x, y, derivatives=False):
        """(u, v) at points (x, y); with `derivatives` also
        (du/dx, du/dy, dv/dx, dv/dy)."""
        Wx, dWx = self.gx.dense(x.reshape(-1))
        Wy, dWy = self.gy.dense(y.reshape(-1))
        out = []
        for c in (0, 1):
            A = Wy @ ctrl[c]
            out.append((A * Wx).sum(1))
        if not derivatives:
            return out[0].reshape(x.shape), out[1].reshape(x.shape)
        d = []
        for c in (0, 1):
            A = Wy @ ctrl[c]
            B = dWy @ ctrl[c]
            d += [(A * dWx).sum(1), (B * Wx).sum(1)]
        return out[0], out[1], d[0], d[1], d[2], d[3]

    def field_fn(self, ctrl, chunk=1 << 18):
        """A callable (X, Y) -> (u, v) for image warping (evaluated in chunks)."""
        def f(X, Y):
            xs, ys = X.reshape(-1), Y.reshape(-1)
            us, vs = [], []
            for b in range(0, xs.numel(), chunk):
                u, v = self.eval(ctrl.to(xs.device), xs[b:b + chunk], ys[b:b + chunk])
                us.append(u)
                vs.append(v)
            return torch.cat(us).reshape(X.shape), torch.cat(vs).reshape(Y.shape)
        return f

    def subset_params(self, ctrl, cx, cy):
        """Affine parameters (n x 6: u, v, theta, ex, ey, gxy) of the field at
        the subset centres."""
        u, v, ux, uy, vx, vy = self.eval(ctrl, cx, cy, derivatives=True)
        f00, f01, f10, f11 = 1.0 + ux, uy, vx, 1.0 + vy
        theta = torch.atan2(f10 - f01, f00 + f11)
        c, s = torch.cos(theta), torch.sin(theta)
        # S = R(-theta) F
        s00 = c * f00 + s * f10
        s11 = -s * f01 + c * f11
        s01 = c * f01 + s * f11
        return torch.stack([u, v, theta, s00 - 1.0, s11 - 1.0, s01], 1)


def fit(schema, def_image, field, cx, cy, iters=200, lr=0.05, lr_final=5e-4, ctrl0=None, objective=0,
        log=None):
    """Fits the control grid of `field` to `schema`'s subsets (centres cx, cy,
    CUDA tensors) on `def_image` by gradient descent (Adam) on the sum of the
    subsets' objective, the step decaying geometrically from `lr` to
    `lr_final` px.  Returns the fitted (2, G, G) control tensor."""
    from dice_b200 import autograd
    dev = def_image.device
    G = field.G
    ctrl = (torch.zeros((2, G, G), dtype=torch.float64, device=dev) if ctrl0 is None
            else ctrl0.detach().clone().to(dev, torch.float64))
    ctrl.requires_grad_(True)
    opt = torch.optim.Adam([ctrl], lr=lr)
    decay = (lr_final / lr) ** (1.0 / max(iters - 1, 1))
    img = def_image.detach()
    for it in range(iters):
        for grp in opt.param_groups:
            grp["lr"] = lr * decay ** it
        opt.zero_grad()
        params = field.subset_params(ctrl, cx, cy)
        val = autograd.subset_objective(params, img, schema, objective)
        loss = val.sum()
        loss.backward()
        opt.step()
        if log is not None:
            log.append(float(loss.detach()))
    return ctrl.detach()


def rms(a):
    return math.sqrt(float((a.double() ** 2).mean()))
