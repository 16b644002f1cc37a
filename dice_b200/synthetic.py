"""Seeded synthetic speckle images and imposed displacement fields.

Stands in for the image pairs of the benchmark configurations (no dataset is
used): Gaussian speckles composited by maximum, optional blur, a deformed
image obtained by sampling the reference at the inverse-mapped position with
the Keys fourth-order kernel (as DICe's apply_transform does,
DICe_ImageUtils.cpp:52-77), plus additive Gaussian noise.  torch is used only
as an array library here (CPU or GPU); the correlation itself runs in
libdicegpu.so.
"""
import math

import numpy as np
import torch


def _gen(seed, device):
    g = torch.Generator(device="cpu")
    g.manual_seed(int(seed))
    return g


def speckle_image(w, h, seed, r_min=2.0, r_max=4.0, coverage=0.5, grey_lo=20.0, grey_hi=230.0,
                  blur_sigma=0.0, device="cpu"):
    """Gaussian speckles (radius r_min..r_max px) until `coverage` of the area,
    intensity grey_lo + (grey_hi - grey_lo) * max_k exp(-d_k^2 / (2 s_k^2)) with
    s_k = r_k / 2, then an optional Gaussian blur.  float32 [h, w]."""
    g = _gen(seed, device)
    r_mean2 = (r_min * r_min + r_min * r_max + r_max * r_max) / 3.0
    n = int(coverage * w * h / (math.pi * r_mean2)) + 1
    cx = torch.rand(n, generator=g, dtype=torch.float64) * (w + 2 * r_max) - r_max
    cy = torch.rand(n, generator=g, dtype=torch.float64) * (h + 2 * r_max) - r_max
    rr = r_min + torch.rand(n, generator=g, dtype=torch.float64) * (r_max - r_min)
    cx, cy, rr = cx.to(device), cy.to(device), rr.to(device)
    R = int(math.ceil(1.5 * r_max))
    off = torch.arange(-R, R + 1, device=device, dtype=torch.float64)
    img = torch.zeros(h * w, dtype=torch.float32, device=device)
    chunk = max(1, 4_000_000 // ((2 * R + 1) ** 2))
    for b in range(0, n, chunk):
        x0 = torch.floor(cx[b:b + chunk])
        y0 = torch.floor(cy[b:b + chunk])
        px = (x0[:, None, None] + off[None, None, :]).expand(-1, off.numel(), -1)
        py = (y0[:, None, None] + off[None, :, None]).expand(-1, -1, off.numel())
        s = (rr[b:b + chunk] / 2.0)[:, None, None]
        d2 = (px - cx[b:b + chunk, None, None]) ** 2 + (py - cy[b:b + chunk, None, None]) ** 2
        val = torch.exp(-d2 / (2.0 * s * s)).to(torch.float32)
        ok = (px >= 0) & (px < w) & (py >= 0) & (py < h)
        idx = (py * w + px)[ok].to(torch.int64)
        img.scatter_reduce_(0, idx, val[ok], reduce="amax")
    img = grey_lo + (grey_hi - grey_lo) * img
    img = img.reshape(h, w)
    if blur_sigma > 0:
        img = gaussian_blur(img, blur_sigma)
    return img


def gaussian_blur(img, sigma):
    k = int(math.ceil(3 * sigma))
    x = torch.arange(-k, k + 1, dtype=torch.float32, device=img.device)
    ker = torch.exp(-x * x / (2 * sigma * sigma))
    ker = ker / ker.sum()
    t = img[None, None]
    t = torch.nn.functional.pad(t, (k, k, 0, 0), mode="replicate")
    t = torch.nn.functional.conv2d(t, ker.view(1, 1, 1, -1))
    t = torch.nn.functional.pad(t, (0, 0, k, k), mode="replicate")
    t = torch.nn.functional.conv2d(t, ker.view(1, 1, -1, 1))
    return t[0, 0]


def _keys_w(t):
    """Keys fourth-order weights for taps -2..3 at fractional offset t (float64)."""
    def k0(s):
        return (4.0 / 3.0) * s ** 3 - (7.0 / 3.0) * s ** 2 + 1.0

    def k1(s):
        return -(7.0 / 12.0) * s ** 3 + 3.0 * s ** 2 - (59.0 / 12.0) * s + 2.5

    def k2(s):
        return (1.0 / 12.0) * s ** 3 - (2.0 / 3.0) * s ** 2 + 1.75 * s - 1.5

    return torch.stack([k2(t + 2), k1(t + 1), k0(t), k0(1 - t), k1(2 - t), k2(3 - t)], dim=-1)


def keys_sample(img, X, Y):
    """Keys-4 samples of img at float64 positions (X, Y); edge-clamped taps."""
    h, w = img.shape
    ix = torch.floor(X)
    iy = torch.floor(Y)
    wx = _keys_w(X - ix)
    wy = _keys_w(Y - iy)
    ix = ix.to(torch.int64)
    iy = iy.to(torch.int64)
    flat = img.reshape(-1).to(torch.float64)
    out = torch.zeros_like(X)
    for m in range(6):
        yy = (iy + (m - 2)).clamp(0, h - 1)
        row = torch.zeros_like(X)
        for n in range(6):
            xx = (ix + (n - 2)).clamp(0, w - 1)
            row += wx[..., n] * flat[yy * w + xx]
        out += wy[..., m] * row
    return out


def warp_image(ref, field, noise_sigma=0.0, seed=0, clip=None, iters=6, block_rows=1024):
    """Deformed image def(x) = ref(X) + noise with x = X + u(X): X found by
    fixed-point iteration X <- x - u(X).  `field(X, Y) -> (u, v)` (float64).
    Rows are processed in blocks of `block_rows` (same result, bounded
    memory for large images)."""
    h, w = ref.shape
    dev = ref.device
    xx = torch.arange(w, device=dev, dtype=torch.float64)
    out = torch.empty((h, w), dtype=torch.float64, device=dev)
    for r0 in range(0, h, block_rows):
        r1 = min(h, r0 + block_rows)
        yy, xb = torch.meshgrid(torch.arange(r0, r1, device=dev, dtype=torch.float64), xx, indexing="ij")
        X, Y = xb.clone(), yy.clone()
        for _ in range(iters):
            u, v = field(X, Y)
            X = xb - u
            Y = yy - v
        out[r0:r1] = keys_sample(ref, X, Y)
    if noise_sigma > 0:
        g = _gen(seed, dev)
        out = out + noise_sigma * torch.randn(out.shape, generator=g, dtype=torch.float64).to(dev)
    if clip is not None:
        out = out.clamp(clip[0], clip[1])
    return out.to(torch.float32)


def grid_points(w, h, subset_size, step):
    """Regular grid of subset centres (create_regular_grid_of_correlation_points,
    DICe_Decomp.cpp:942-951): x from subset_size-1 by `step` while
    x < w - subset_size; row-major order."""
    xs = list(range(subset_size - 1, w - subset_size, step))
    ys = list(range(subset_size - 1, h - subset_size, step))
    X, Y = np.meshgrid(np.asarray(xs, np.float64), np.asarray(ys, np.float64))
    return X.ravel(), Y.ravel()


def init_fields(cx, cy, quadratic=False):
    from .abi import FIELD_STRIDE, F_COORD_X, F_COORD_Y, F_QUAD_A
    f = np.zeros((len(cx), FIELD_STRIDE), np.float64)
    f[:, F_COORD_X] = cx
    f[:, F_COORD_Y] = cy
    if quadratic:
        f[:, F_QUAD_A + 0] = 1.0
        f[:, F_QUAD_A + 7] = 1.0
    return f


# ---- the benchmark configurations (seeded stand-ins) -----------------------
def config1(device="cpu", w=512, h=512):
    """512^2 speckle pair: radius 2-4, 50 % coverage, grey 20-230, blur 0.8;
    translation u=0.37, v=-1.21 resampled with Keys-4, noise sigma 2; seed 1."""
    ref = speckle_image(w, h, seed=1, r_min=2, r_max=4, grey_lo=20, grey_hi=230, blur_sigma=0.8,
                        device=device)
    deff = warp_image(ref, lambda X, Y: (torch.full_like(X, 0.37), torch.full_like(Y, -1.21)),
                      noise_sigma=2.0, seed=101, clip=(0.0, 255.0))
    return ref, deff


def config2_field(k, nframes=10):
    """Frame k of the sinusoidal field u = 0.5 sin(2 pi x/128), v = 0.3 cos(2 pi y/96)
    plus 0.2 % uniform strain, scaled by k/nframes."""
    s = float(k) / float(nframes)

    def f(X, Y):
        u = 0.5 * torch.sin(2 * math.pi * X / 128.0) + 0.002 * X
        v = 0.3 * torch.cos(2 * math.pi * Y / 96.0) + 0.002 * Y
        return s * u, s * v
    return f


def _convex_hull(pts):
    pts = sorted(map(tuple, pts))
    if len(pts) < 3:
        return pts

    def cross(o, a, b):
        return (a[0] - o[0]) * (b[1] - o[1]) - (a[1] - o[1]) * (b[0] - o[0])
    lo, hi = [], []
    for p in pts:
        while len(lo) >= 2 and cross(lo[-2], lo[-1], p) <= 0:
            lo.pop()
        lo.append(p)
    for p in reversed(pts):
        while len(hi) >= 2 and cross(hi[-2], hi[-1], p) <= 0:
            hi.pop()
        hi.append(p)
    return lo[:-1] + hi[:-1]


def mixed_subsets(w, h, n, seed, margin=40):
    """Seeded arbitrary-shape subsets: circles (radius 7-25 px), ellipses with
    60 x 8 px axes at random orientation, and random convex polygons, 150-2000
    pixels each, as CSR pixel lists sorted by (y, x) like the reference's
    conformal subsets (DICe_Subset.cpp:115-142).  Returns
    (cx, cy, offsets, px, py, kind, minor_extent) with kind 0 circle,
    1 ellipse, 2 polygon."""
    rng = np.random.default_rng(seed)
    cx = rng.integers(margin, w - margin, n)
    cy = rng.integers(margin, h - margin, n)
    kind = rng.integers(0, 3, n)
    offs = [0]
    pxs, pys, minor = [], [], []
    for i in range(n):
        x0, y0 = int(cx[i]), int(cy[i])
        if kind[i] == 0:
            r = rng.uniform(7.0, 25.0)
            R = int(np.ceil(r))
            yy, xx = np.mgrid[-R:R + 1, -R:R + 1]
            m = xx * xx + yy * yy <= r * r
            minor.append(2 * r)
        elif kind[i] == 1:
            phi = rng.uniform(0, np.pi)
            R = 31
            yy, xx = np.mgrid[-R:R + 1, -R:R + 1]
            a = (xx * np.cos(phi) + yy * np.sin(phi)) / 30.0
            b = (-xx * np.sin(phi) + yy * np.cos(phi)) / 4.0
            m = a * a + b * b <= 1.0
            minor.append(8.0)
        else:
            rr = rng.uniform(10.0, 25.0)
            ang = rng.uniform(0, 2 * np.pi, 9)
            rad = rr * np.sqrt(rng.uniform(0.3, 1.0, 9))
            hull = _convex_hull(np.stack([rad * np.cos(ang), rad * np.sin(ang)], 1))
            R = int(np.ceil(rr)) + 1
            yy, xx = np.mgrid[-R:R + 1, -R:R + 1]
            m = np.ones_like(xx, dtype=bool)
            for k in range(len(hull)):
                ax, ay = hull[k]
                bx, by = hull[(k + 1) % len(hull)]
                m &= (bx - ax) * (yy - ay) - (by - ay) * (xx - ax) >= 0
            ext = [np.ptp(xx[m]) + 1 if m.any() else 0, np.ptp(yy[m]) + 1 if m.any() else 0]
            minor.append(float(min(ext)))
        ys, xs = np.nonzero(m)
        order = np.lexsort((xs, ys))
        pys.append((ys[order] + y0 - R).astype(np.int32))
        pxs.append((xs[order] + x0 - R).astype(np.int32))
        offs.append(offs[-1] + int(m.sum()))
    return (cx.astype(np.float64), cy.astype(np.float64), np.asarray(offs, np.int32),
            np.concatenate(pxs), np.concatenate(pys), kind, np.asarray(minor))


def config3_field(w, h, angle_deg=1.5, shear=0.005):
    """Rigid rotation about the image centre plus simple shear (x += shear * (Y - cy))."""
    th = np.deg2rad(angle_deg)
    c, s = float(np.cos(th)), float(np.sin(th))
    xc, yc = (w - 1) / 2.0, (h - 1) / 2.0

    def f(X, Y):
        dx = X - xc + shear * (Y - yc)
        dy = Y - yc
        x = xc + c * dx - s * dy
        y = yc + s * dx + c * dy
        return x - X, y - Y
    return f


def config5_field(h, jump=2.0, strain=0.003):
    """Mode-I crack: a 2 px opening across the horizontal line y = h/2 plus a
    linear far field of 0.3 % strain."""
    yc = h / 2.0

    def f(X, Y):
        u = strain * X
        v = strain * Y + torch.where(Y >= yc, torch.full_like(Y, jump / 2.0), torch.full_like(Y, -jump / 2.0))
        return u, v
    return f


def config3(device="cpu", w=4096, h=3000, n=50000, seed=3, noise_sigma=1.0):
    """4096 x 3000 speckle pair under a 1.5 degree rotation about the centre
    plus 0.5 % shear, and `n` seeded mixed subsets (mixed_subsets).  Returns
    (ref, def, field, subsets) with subsets = (cx, cy, offsets, px, py, kind,
    minor_extent)."""
    ref = speckle_image(w, h, seed=seed, r_min=2.0, r_max=4.0, grey_lo=20.0, grey_hi=230.0,
                        blur_sigma=0.8, device=device)
    field = config3_field(w, h)
    deff = warp_image(ref, field, noise_sigma=noise_sigma, seed=seed + 300, clip=(0.0, 255.0))
    return ref, deff, field, mixed_subsets(w, h, n, seed=seed + 30)


def config5(device="cpu", w=8192, h=8192, nframes=8, jump=2.0, strain=0.003, count=None, seed=5,
            noise_sigma=1.0):
    """8192^2 speckle sequence of a mode-I crack: frame k (1..nframes) opens
    the jump across y = h/2 to jump * k / nframes px on top of a linear far
    field of strain * k / nframes.  Returns (ref, first `count` frames)."""
    ref = speckle_image(w, h, seed=seed, r_min=2.0, r_max=4.0, grey_lo=20.0, grey_hi=230.0,
                        blur_sigma=0.8, device=device)
    count = nframes if count is None else count
    frames = [warp_image(ref, config5_field(h, jump * (k + 1) / nframes, strain * (k + 1) / nframes),
                         noise_sigma=noise_sigma, seed=seed + 500 + k, clip=(0.0, 255.0))
              for k in range(count)]
    return ref, frames


def config4(device="cpu", w=1024, h=1024, ncontrol=16, ctrl_sigma=0.8, noise_sigma=1.0, seed=4):
    """1024^2 speckle pair whose field is a seeded 16 x 16 cubic B-spline
    control grid with N(0, 0.8 px) control displacements.  Returns
    (ref, def, field, ctrl) with ctrl the (2, G, G) control tensor."""
    from dice_b200.bspline import BSplineField
    ref = speckle_image(w, h, seed=seed, r_min=2.0, r_max=4.0, grey_lo=20.0, grey_hi=230.0,
                        blur_sigma=0.8, device=device)
    g = _gen(seed + 1000, "cpu")
    ctrl = (ctrl_sigma * torch.randn((2, ncontrol, ncontrol), generator=g, dtype=torch.float64)).to(device)
    field = BSplineField(w, h, ncontrol)
    deff = warp_image(ref, field.field_fn(ctrl), noise_sigma=noise_sigma, seed=seed + 100, clip=(0.0, 255.0))
    return ref, deff, field, ctrl


def config2(device="cpu", w=2048, h=2048, nframes=10, count=None):
    """2048^2 16-bit-range speckle image (radius 3-5) and the first `count`
    (default all `nframes`) deformed frames of the sequence."""
    ref = speckle_image(w, h, seed=2, r_min=3, r_max=5, grey_lo=1000.0, grey_hi=64000.0,
                        blur_sigma=0.8, device=device)
    count = nframes if count is None else count
    frames = [warp_image(ref, config2_field(k + 1, nframes), noise_sigma=50.0, seed=200 + k,
                         clip=(0.0, 65535.0)) for k in range(count)]
    return ref, frames
