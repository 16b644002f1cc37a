"""ctypes binding of the CPU oracle (oracle/libdiceoracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py as the checker / CPU baseline.  The product
(dice_b200, libdicegpu.so) never imports it.
"""
import ctypes
import os

import numpy as np

from dice_b200.abi import Params, FIELD_STRIDE, UNCERTAINTY_STRIDE, TRACKING_ROUTINE, shape_array

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdiceoracle.so")
_lib = None


class use_library:
    """Context manager: route the oracle calls to another build of it (for
    instance libdiceoracle_meanfp64.so, the rounding-sensitivity variant)."""

    def __init__(self, name):
        self.path = os.path.join(_HERE, name)

    def __enter__(self):
        global LIB_PATH, _lib
        self._saved = (LIB_PATH, _lib)
        LIB_PATH, _lib = self.path, None
        return self

    def __exit__(self, *exc):
        global LIB_PATH, _lib
        LIB_PATH, _lib = self._saved
        return False


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(Params)
        vp, ci = ctypes.c_void_p, ctypes.c_int
        L.oracle_execute_frame.restype = ci
        L.oracle_execute_frame.argtypes = [P, ci, ci, vp, vp, ci, vp, vp, vp, vp, vp, ci, ci, vp, vp, vp, vp]
        L.oracle_gradients.restype = ci
        L.oracle_gradients.argtypes = [ci, ci, vp, ci, vp, vp]
        L.oracle_gauss_filter.restype = ci
        L.oracle_gauss_filter.argtypes = [ci, ci, vp, vp, ci]
        L.oracle_interpolate.restype = ci
        L.oracle_interpolate.argtypes = [ci, ci, ci, vp, vp, vp, ci, vp, vp, vp, vp]
        L.oracle_gamma.restype = ci
        L.oracle_gamma.argtypes = [P, ci, ci, vp, vp, ci, vp, vp]
        L.oracle_gn_system.restype = ci
        L.oracle_gn_system.argtypes = [P, ci, ci, vp, vp, ci, vp, vp, vp]
        L.oracle_objective.restype = ci
        L.oracle_objective.argtypes = [P, ci, ci, vp, vp, ci, vp, ci, vp, vp, vp, vp]
        L.oracle_default_params.restype = ci
        L.oracle_default_params.argtypes = [P]
        L.oracle_map.restype = ci
        L.oracle_map.argtypes = [P, vp, ci, vp, ctypes.c_float, ctypes.c_float, vp]
        L.oracle_rasterize.restype = ci
        L.oracle_rasterize.argtypes = [ci, ci, vp, vp, vp, vp, ci, vp, vp, vp]
        L.oracle_execute_frame_shapes.restype = ci
        L.oracle_execute_frame_shapes.argtypes = [P, ci, ci, vp, vp, ci, vp, ci, vp, vp, vp, vp, vp, vp, ci, ci,
                                                  vp, vp, ci]
        L.oracle_vsg_strain.restype = ci
        L.oracle_vsg_strain.argtypes = [ci, vp, ci, vp, vp]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _subset_flags(n, force_simplex, skip_solve):
    """Per-subset flag bytes of the oracle: bit 0 forces the simplex, bit 1
    skips the solve."""
    if force_simplex is None and skip_solve is None:
        return None
    f = np.zeros(n, np.uint8)
    if force_simplex is not None:
        f |= (np.asarray(force_simplex) != 0).astype(np.uint8)
    if skip_solve is not None:
        f |= 2 * (np.asarray(skip_solve) != 0).astype(np.uint8)
    return np.ascontiguousarray(f)


def execute_frame(params, ref, deff, fields, first_frame=True, nthreads=1, offsets=None,
                  px=None, py=None, force_simplex=None, counters=False, uncertainty=None, neighbors=None,
                  skip_solve=None):
    """One frame over all subsets; updates `fields` (n x FIELD_STRIDE float64) in place.
    `uncertainty` (n x UNCERTAINTY_STRIDE float64, optional) receives the
    uncertainty fields of every converged Gauss-Newton solve.  `neighbors`
    (NEIGHBOR_ID per subset) serve params.initialization_method.
    `skip_solve` (per subset, non-zero: skip) only evaluates those subsets at
    their initial guess (FRAME_SKIPPED)."""
    if neighbors is not None:
        neighbors = np.ascontiguousarray(neighbors, dtype=np.int32)
    if uncertainty is not None:
        assert uncertainty.dtype == np.float64 and uncertainty.flags.c_contiguous
        assert uncertainty.shape == (fields.shape[0], UNCERTAINTY_STRIDE)
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    deff = np.ascontiguousarray(deff, dtype=np.float32)
    assert fields.dtype == np.float64 and fields.flags.c_contiguous and fields.shape[1] == FIELD_STRIDE
    h, w = ref.shape
    n = fields.shape[0]
    if offsets is not None:
        offsets = np.ascontiguousarray(offsets, dtype=np.int32)
        px = np.ascontiguousarray(px, dtype=np.int32)
        py = np.ascontiguousarray(py, dtype=np.int32)
    force_simplex = _subset_flags(n, force_simplex, skip_solve)
    gn = np.zeros(n, np.int32) if counters else None
    sx = np.zeros(n, np.int32) if counters else None
    rc = lib().oracle_execute_frame(ctypes.byref(params), w, h, _ptr(ref), _ptr(deff), n,
                                    _ptr(fields), _ptr(offsets), _ptr(px), _ptr(py),
                                    _ptr(force_simplex), 1 if first_frame else 0, nthreads,
                                    _ptr(gn), _ptr(sx), _ptr(uncertainty), _ptr(neighbors))
    if rc != 0:
        raise RuntimeError("oracle_execute_frame failed: %d" % rc)
    if counters:
        return gn, sx
    return None


def shape_map(params, field_row, xy, cx, cy):
    """Local_Shape_Function::map of points xy (n x 2) about (cx, cy)."""
    f = np.ascontiguousarray(field_row, dtype=np.float64)
    xy = np.ascontiguousarray(xy, dtype=np.float32).reshape(-1, 2)
    out = np.zeros_like(xy)
    rc = lib().oracle_map(ctypes.byref(params), _ptr(f), xy.shape[0], _ptr(xy), cx, cy, _ptr(out))
    assert rc == 0
    return out


def rasterize(n, shapes, vx=None, vy=None, fields=None, square_size=0):
    """Pixel lists (offsets, px, py) of n subsets from their shapes
    (dice_b200.abi.Shape), as get_owned_pixels builds them; subsets without
    boundary shapes are squares of square_size about the field rows'
    coordinates (when fields are given)."""
    arr = shape_array(list(shapes))
    x = np.ascontiguousarray(vx if vx is not None else [0], dtype=np.int32)
    y = np.ascontiguousarray(vy if vy is not None else [0], dtype=np.int32)
    f = None if fields is None else np.ascontiguousarray(fields, dtype=np.float64)
    offs = np.zeros(n + 1, np.int32)
    sp = ctypes.cast(arr, ctypes.c_void_p)
    rc = lib().oracle_rasterize(n, len(arr), sp, _ptr(x), _ptr(y), _ptr(f), square_size, _ptr(offs), None, None)
    assert rc == 0, rc
    px = np.zeros(max(int(offs[-1]), 1), np.int32)
    py = np.zeros_like(px)
    rc = lib().oracle_rasterize(n, len(arr), sp, _ptr(x), _ptr(y), _ptr(f), square_size, _ptr(offs),
                                _ptr(px), _ptr(py))
    assert rc == 0, rc
    return offs, px[:offs[-1]], py[:offs[-1]]


def execute_frame_shapes(params, ref, deff, fields, shapes, vx=None, vy=None, block_offsets=None,
                         block_ids=None, force_simplex=None, first_frame=True, nthreads=1, evolution=None,
                         frame_index=0, skip_solve=None):
    """Schema::execute_correlation over subsets defined by shapes with
    obstructions and blocking subsets; updates `fields` in place.  With
    params.use_subset_evolution, `evolution` is a dict carried across the
    frames of a sequence (the per-pixel state) and frame_index counts them."""
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    deff = np.ascontiguousarray(deff, dtype=np.float32)
    assert fields.dtype == np.float64 and fields.flags.c_contiguous
    h, w = ref.shape
    n = fields.shape[0]
    arr = shape_array(list(shapes))
    x = np.ascontiguousarray(vx if vx is not None else [0], dtype=np.int32)
    y = np.ascontiguousarray(vy if vy is not None else [0], dtype=np.int32)
    bo = None if block_offsets is None else np.ascontiguousarray(block_offsets, dtype=np.int32)
    bi = None if block_ids is None else np.ascontiguousarray(block_ids if len(block_ids) else [0], dtype=np.int32)
    fs = _subset_flags(n, force_simplex, skip_solve)
    pf = pv = None
    if evolution is not None and params.use_subset_evolution and params.correlation_routine == TRACKING_ROUTINE:
        if "flag" not in evolution:
            total = int(rasterize(n, shapes, vx, vy, fields, params.subset_size)[0][-1])
            # the lists keep the excluded pixels: size them from the boundaries alone
            bounds = [sh for sh in shapes if sh.role == 0]
            total = int(rasterize(n, bounds, vx, vy, fields, params.subset_size)[0][-1]) if bounds else total
            evolution["flag"] = np.zeros(max(total, 1), np.uint8)
            evolution["f"] = np.zeros(max(total, 1), np.float32)
        pf, pv = evolution["flag"], evolution["f"]
    rc = lib().oracle_execute_frame_shapes(ctypes.byref(params), w, h, _ptr(ref), _ptr(deff), n, _ptr(fields),
                                           len(arr), ctypes.cast(arr, ctypes.c_void_p), _ptr(x), _ptr(y),
                                           _ptr(bo), _ptr(bi), _ptr(fs), int(first_frame), nthreads, _ptr(pf),
                                           _ptr(pv), int(frame_index))
    if rc != 0:
        raise RuntimeError("oracle_execute_frame_shapes: %d" % rc)
    return fields


def execute_sequence(params, ref, frames, fields, run=None, evolution=None):
    """Schema::execute_correlation over a sequence of deformed frames
    (DICe_Main.cpp:324-360).  With params.use_incremental_formulation, every
    frame after the first correlates against the previous deformed frame
    (set_ref_image(prev_img()), :326-328), starts with DISPLACEMENT_X / _Y
    at 0 and ends with them accumulated (DICe_Schema.cpp:1671-1675,
    1775-1789; the first frame is not accumulated), and the tracking
    routine re-reads every reference intensity, turned-on pixels included
    (:1757-1759).  `run(ref, deff, fields, k)` runs frame k (default: the
    square / list path); returns the field rows after each frame."""
    if run is None:
        def run(r, d, f, k):
            execute_frame(params, r, d, f, first_frame=(k == 0))
    incr = params.use_incremental_formulation != 0
    acc = np.zeros((fields.shape[0], 2))
    rows = []
    cur = ref
    for k, d in enumerate(frames):
        if incr and k > 0:
            cur = frames[k - 1]
            fields[:, 2] = 0.0   # DISPLACEMENT_X
            fields[:, 3] = 0.0   # DISPLACEMENT_Y
            if evolution and "flag" in evolution and params.correlation_routine == TRACKING_ROUTINE:
                evolution["flag"][evolution["flag"] == 2] = 1
        run(cur, d, fields, k)
        if incr and k > 0:
            acc += fields[:, 2:4]
            fields[:, 2:4] = acc
        rows.append(fields.copy())
    return rows


def vsg_strain(fields, window):
    """VSG_Strain_Post_Processor on the field rows: (n x 7 values, failed flags)."""
    f = np.ascontiguousarray(fields, dtype=np.float64)
    n = f.shape[0]
    out = np.zeros((n, 7), np.float64)
    failed = np.zeros(n, np.int32)
    rc = lib().oracle_vsg_strain(n, _ptr(f), int(window), _ptr(out), _ptr(failed))
    assert rc == 0, rc
    return out, failed


def gauss_filter(img, mask_size=7):
    img = np.ascontiguousarray(img, dtype=np.float32)
    h, w = img.shape
    out = np.zeros_like(img)
    rc = lib().oracle_gauss_filter(w, h, _ptr(img), _ptr(out), mask_size)
    assert rc == 0, rc
    return out


def gradients(img, method=0):
    img = np.ascontiguousarray(img, dtype=np.float32)
    h, w = img.shape
    gx = np.zeros_like(img)
    gy = np.zeros_like(img)
    rc = lib().oracle_gradients(w, h, _ptr(img), method, _ptr(gx), _ptr(gy))
    assert rc == 0
    return gx, gy


def interpolate(method, img, xy, gx=None, gy=None):
    img = np.ascontiguousarray(img, dtype=np.float32)
    xy = np.ascontiguousarray(xy, dtype=np.float32).reshape(-1, 2)
    h, w = img.shape
    n = xy.shape[0]
    oi = np.zeros(n, np.float32)
    ogx = np.zeros(n, np.float32) if gx is not None else None
    ogy = np.zeros(n, np.float32) if gy is not None else None
    if gx is not None:
        gx = np.ascontiguousarray(gx, dtype=np.float32)
        gy = np.ascontiguousarray(gy, dtype=np.float32)
    rc = lib().oracle_interpolate(method, w, h, _ptr(img), _ptr(gx), _ptr(gy), n, _ptr(xy),
                                  _ptr(oi), _ptr(ogx), _ptr(ogy))
    assert rc == 0
    return oi, ogx, ogy


def gamma(params, ref, deff, fields):
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    deff = np.ascontiguousarray(deff, dtype=np.float32)
    h, w = ref.shape
    out = np.zeros(fields.shape[0], np.float64)
    rc = lib().oracle_gamma(ctypes.byref(params), w, h, _ptr(ref), _ptr(deff), fields.shape[0],
                            _ptr(fields), _ptr(out))
    assert rc == 0
    return out


def objective(params, ref, deff, fields, op):
    """op 0 computeUpdateFast / 1 computeUpdateRobust: updates `fields` in place
    and returns (iterations, status); op 2 sigma: returns (sigma, noise)."""
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    deff = np.ascontiguousarray(deff, dtype=np.float32)
    assert fields.dtype == np.float64 and fields.flags.c_contiguous
    h, w = ref.shape
    n = fields.shape[0]
    it = np.zeros(n, np.int32)
    st = np.zeros(n, np.int32)
    sg = np.zeros(n, np.float64)
    no = np.zeros(n, np.float64)
    rc = lib().oracle_objective(ctypes.byref(params), w, h, _ptr(ref), _ptr(deff), n, _ptr(fields), op,
                                _ptr(it), _ptr(st), _ptr(sg), _ptr(no))
    assert rc == 0, rc
    return (sg, no) if op == 2 else (it, st)


def gn_system(params, ref, deff, fields, nparams):
    """(H, q) of the Gauss-Newton system at the parameters of each field row."""
    ref = np.ascontiguousarray(ref, dtype=np.float32)
    deff = np.ascontiguousarray(deff, dtype=np.float32)
    f = np.ascontiguousarray(fields, dtype=np.float64)
    h, w = ref.shape
    n = f.shape[0]
    H = np.zeros((n, nparams, nparams))
    q = np.zeros((n, nparams))
    rc = lib().oracle_gn_system(ctypes.byref(params), w, h, _ptr(ref), _ptr(deff), n, _ptr(f),
                                _ptr(H), _ptr(q))
    assert rc == 0, rc
    return H, q
