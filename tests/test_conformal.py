"""Conformal subsets: pixel lists built from circle / rectangle / polygon shapes.

The oracle restates get_owned_pixels (DICe_Shape.cpp:136-420) and the
conformal Subset constructor (DICe_Subset.cpp:115-142), and is pinned to the
reference's own conformal-subset image (DICe_TestSubset.cpp:248-300: two
polygons minus an 11 x 7 rectangle, written by Subset::write_image over the
subset's bounding box and stored as images/conformal.rawi).  In that image a
pixel is non-zero exactly when it lies in the union of the polygons; the
excluded pixels, which the reference keeps as inactive, are all written with
one grey (131).  The device rasterizer must equal the oracle pixel for pixel,
and a correlation over device-built lists must equal one over the same lists
uploaded from the host.
"""
import os

import numpy as np
import pytest

from dice_b200 import abi
from dice_b200 import synthetic as syn
from oracle import oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_gold.npz"))

VX = [940, 951, 964, 980, 959, 982, 1000, 991, 978]
VY = [422, 399, 410, 413, 432, 426, 428, 456, 445]
REF_SHAPES = [abi.polygon(0, 0, 5), abi.polygon(0, 5, 4), abi.rectangle(0, 955, 423, 11, 7, role=1)]


def _mask(px, py, x0, y0, shape):
    m = np.zeros(shape, bool)
    m[py - y0, px - x0] = True
    return m


def test_oracle_conformal_subset_matches_reference_image():
    gold = GOLD["conformal_subset_image"]
    offs, px, py = O.rasterize(1, REF_SHAPES[:2], VX, VY)
    x0, y0 = px.min(), py.min()          # the image spans the subset's bounding box
    assert gold.shape == (py.max() - y0 + 1, px.max() - x0 + 1)
    union = _mask(px, py, x0, y0, gold.shape)
    assert np.array_equal(union, gold != 0)
    # with the rectangle excluded: the removed pixels are the inactive ones
    offs_e, ex, ey = O.rasterize(1, REF_SHAPES, VX, VY)
    owned = _mask(ex, ey, x0, y0, gold.shape)
    excluded = union & ~owned
    assert excluded.sum() == 77
    assert np.all(gold[excluded] == 131.0)
    ys, xs = np.nonzero(excluded)
    assert xs.min() + x0 >= 950 and xs.max() + x0 <= 960
    assert ys.min() + y0 >= 420 and ys.max() + y0 <= 426
    assert offs_e[-1] == offs[-1] - 77
    # (y, x) order
    assert np.array_equal(np.lexsort((ex, ey)), np.arange(len(ex)))


def test_oracle_basic_shapes():
    offs, px, py = O.rasterize(1, [abi.rectangle(0, 10, 20, 5, 3)])
    assert offs[-1] == 15
    assert (px.min(), px.max(), py.min(), py.max()) == (8, 12, 19, 21)
    offs, px, py = O.rasterize(1, [abi.circle(0, 50, 50, 3.0)])
    assert offs[-1] == 29                 # integer points with dx^2 + dy^2 <= 9
    assert np.all((px - 50) ** 2 + (py - 50) ** 2 <= 9)
    # union of two overlapping shapes counts shared pixels once, a hole removes
    offs, px, py = O.rasterize(1, [abi.rectangle(0, 10, 10, 6, 6), abi.rectangle(0, 12, 10, 6, 6),
                                   abi.circle(0, 11, 10, 1.0, role=1)])
    assert offs[-1] == 8 * 6 - 5
    # negative coordinates clamp to 0 after ordering (the constructor's rule)
    offs, px, py = O.rasterize(1, [abi.rectangle(0, 0, 0, 4, 4)])
    assert offs[-1] == 16 and px.min() == 0 and py.min() == 0
    # a subset without boundary shapes is empty
    offs, px, py = O.rasterize(2, [abi.circle(1, 20, 20, 2.0)])
    assert offs[1] == 0 and offs[2] > 0


def _random_shapes(n, seed):
    rng = np.random.default_rng(seed)
    shapes, vx, vy = [], [], []
    for i in range(n):
        cx, cy = int(rng.integers(30, 900)), int(rng.integers(30, 700))
        for _ in range(int(rng.integers(1, 3))):
            k = int(rng.integers(0, 3))
            ox, oy = cx + int(rng.integers(-6, 7)), cy + int(rng.integers(-6, 7))
            if k == 0:
                shapes.append(abi.circle(i, ox, oy, float(rng.uniform(2.0, 17.0))))
            elif k == 1:
                shapes.append(abi.rectangle(i, ox, oy, int(rng.integers(1, 30)), int(rng.integers(1, 30))))
            else:
                m = int(rng.integers(3, 9))
                ang = np.sort(rng.uniform(0, 2 * np.pi, m))
                rad = rng.uniform(4.0, 18.0, m)
                shapes.append(abi.polygon(i, len(vx), m))
                vx += list(np.round(ox + rad * np.cos(ang)).astype(int))
                vy += list(np.round(oy + rad * np.sin(ang)).astype(int))
        if rng.random() < 0.4:
            shapes.append(abi.circle(i, cx, cy, float(rng.uniform(1.0, 5.0)), role=1))
        if rng.random() < 0.2:
            shapes.append(abi.rectangle(i, cx + 3, cy - 2, 5, 4, role=1))
    perm = rng.permutation(len(shapes))     # shapes need not arrive grouped by subset
    return [shapes[j] for j in perm], np.asarray(vx, np.int32), np.asarray(vy, np.int32)


def _gpu():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def _device_lists(n, shapes, vx, vy):
    from dice_b200.schema import Schema
    with Schema(abi.default_params(subset_size=0)) as s:
        s.set_ref_image(np.zeros((64, 64), np.float32))
        s.set_subsets(np.full(n, 32.0), np.full(n, 32.0))
        s.set_subset_shapes(shapes, vx, vy)
        out = s.subset_pixels()
        assert s.device_status() == 0
    return out


@pytest.mark.gpu
def test_gpu_rasterizer_reference_shapes():
    _gpu()
    want = O.rasterize(1, REF_SHAPES, VX, VY)
    got = _device_lists(1, REF_SHAPES, np.asarray(VX, np.int32), np.asarray(VY, np.int32))
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [1, 2])
def test_gpu_rasterizer_matches_oracle_random_shapes(seed):
    _gpu()
    shapes, vx, vy = _random_shapes(600, seed)
    want = O.rasterize(600, shapes, vx, vy)
    got = _device_lists(600, shapes, vx, vy)
    for a, b in zip(got, want):
        assert np.array_equal(a, b)


@pytest.mark.gpu
def test_gpu_rasterizer_rejects_bad_shapes():
    _gpu()
    from dice_b200.schema import Schema
    with Schema(abi.default_params(subset_size=0)) as s:
        s.set_ref_image(np.zeros((64, 64), np.float32))
        s.set_subsets(np.full(2, 32.0), np.full(2, 32.0))
        for bad in ([abi.circle(2, 5, 5, 2.0)],                    # subset out of range
                    [abi.circle(0, 5, 5, 2.0, role=3)],            # unknown role
                    [abi.circle(0, 5, 5, -1.0)],                   # negative radius
                    [abi.rectangle(0, 5, 5, 40000, 3)],            # extent above 32768
                    [abi.polygon(0, 0, 2)],                        # fewer than 3 vertices
                    [abi.circle(0, 0, 0, 9000.0), abi.circle(0, 30000, 0, 9000.0)]):   # box too wide
            with pytest.raises(Exception):
                s.set_subset_shapes(bad, [0, 1, 2], [0, 1, 2])


@pytest.mark.gpu
def test_correlation_on_device_built_subsets_equals_host_lists():
    _gpu()
    from dice_b200.schema import Schema
    ref, deff = syn.config1(w=480, h=360)
    ref, deff = ref.numpy(), deff.numpy()
    shapes, vx, vy = _random_shapes(240, 7)
    # subsets centred on their first boundary shape's box, well inside the image
    offs, px, py = O.rasterize(240, shapes, vx, vy)
    keep = []
    cx, cy = np.zeros(240), np.zeros(240)
    for i in range(240):
        x, y = px[offs[i]:offs[i + 1]], py[offs[i]:offs[i + 1]]
        if len(x) >= 60 and x.min() > 12 and y.min() > 12 and x.max() < 468 and y.max() < 348:
            keep.append(i)
            cx[i], cy[i] = np.round(x.mean()), np.round(y.mean())
    keep = np.asarray(keep)
    remap = {int(i): j for j, i in enumerate(keep)}
    sub = [abi.Shape(s.kind, remap[s.subset], s.role, s.cx, s.cy, s.width, s.height, s.radius,
                     s.vertex_offset, s.vertex_count) for s in shapes if s.subset in remap]
    lists = O.rasterize(len(keep), sub, vx, vy)
    p = abi.default_params(subset_size=0, enable_rotation=1, fast_solver_tolerance=1e-5)
    f = syn.init_fields(cx[keep], cy[keep])
    out = []
    for how in ("shapes", "lists"):
        with Schema(p) as s:
            s.set_ref_image(ref)
            s.set_fields(f)
            if how == "shapes":
                s.set_subset_shapes(sub, vx, vy)
            else:
                s.set_subset_pixels(*lists)
            s.set_def_image(deff)
            s.execute_correlation()
            out.append(s.fields())
    assert np.array_equal(out[0], out[1])
    assert np.mean(out[0][:, abi.F_STATUS] < 2) > 0.8
