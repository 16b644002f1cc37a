"""DICe subset files through the C ABI (include/dicegpu_subset_file.h).

`SubsetFile` mirrors what read_subset_file (DICe_Parser.cpp:1098-1650)
returns in Subset_File_Info: the coordinates, the conformal definitions as
shape rows, the blocking lists, the FORCE_SIMPLEX set and the seeds; `apply`
hands them to a Schema the way Schema::initialize does with a subset file
(DICe_Schema.cpp:1025-1145).
"""
import ctypes

import numpy as np

from . import abi

SEED_DISPLACEMENT, SEED_NORMAL_STRAIN, SEED_SHEAR_STRAIN, SEED_ROTATION = 1, 2, 4, 8
FEATURE_SKIP_SOLVE, FEATURE_OPTICAL_FLOW, FEATURE_PATH_FILE, FEATURE_MOTION_WINDOW, FEATURE_TEST_MOTION = (
    1, 2, 4, 8, 16)


class Info(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int32) for k in ("n_subsets", "n_shapes", "n_vertices", "n_blocking_ids",
                                                "n_conformal", "region_of_interest", "n_seeds", "n_unsupported",
                                                "n_skip_solve_ids")]


class SubsetFileError(ValueError):
    pass


def _vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class SubsetFile:
    """A parsed subset file.  `text` (str) or `path`; width / height bound the
    coordinates as the reference checks them (-1: unchecked)."""

    def __init__(self, path=None, text=None, width=-1, height=-1):
        self.lib = abi.load_library()
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        if text is not None:
            raw = text.encode() if isinstance(text, str) else bytes(text)
            rc = self.lib.dicegpu_subset_file_parse(raw, len(raw), width, height, ctypes.byref(h), err, 512)
        else:
            rc = self.lib.dicegpu_subset_file_read(str(path).encode(), width, height, ctypes.byref(h), err, 512)
        if rc != 0:
            raise SubsetFileError(err.value.decode() or abi.ERR_NAMES.get(rc, str(rc)))
        self.h = h
        info = Info()
        abi.check(self.lib.dicegpu_subset_file_get_info(self.h, ctypes.byref(info)), "subset_file_get_info")
        self.info = info
        n = info.n_subsets
        self.coordinates = np.zeros((n, 2), np.float64)
        if n:
            abi.check(self.lib.dicegpu_subset_file_coordinates(self.h, _vp(self.coordinates)), "coordinates")
        arr = (abi.Shape * max(info.n_shapes, 1))()
        vx = np.zeros(max(info.n_vertices, 1), np.int32)
        vy = np.zeros_like(vx)
        if info.n_shapes:
            abi.check(self.lib.dicegpu_subset_file_shapes(self.h, ctypes.cast(arr, ctypes.c_void_p), _vp(vx), _vp(vy)),
                      "shapes")
        self.shapes = list(arr)[:info.n_shapes]
        self.vx, self.vy = vx[:info.n_vertices], vy[:info.n_vertices]
        offs = np.zeros(n + 1, np.int32)
        ids = np.zeros(max(info.n_blocking_ids, 1), np.int32)
        abi.check(self.lib.dicegpu_subset_file_blocking(self.h, _vp(offs), _vp(ids)), "blocking")
        self.blocking = [list(ids[offs[i]:offs[i + 1]]) for i in range(n)]
        self.force_simplex = np.zeros(max(n, 1), np.uint8)
        self.seed_values = np.zeros((max(n, 1), 6), np.float64)
        self.seed_flags = np.zeros(max(n, 1), np.uint8)
        self.features = np.zeros(max(n, 1), np.uint8)
        if n:
            abi.check(self.lib.dicegpu_subset_file_force_simplex(self.h, _vp(self.force_simplex)), "force_simplex")
            abi.check(self.lib.dicegpu_subset_file_seeds(self.h, _vp(self.seed_values), _vp(self.seed_flags)), "seeds")
            abi.check(self.lib.dicegpu_subset_file_features(self.h, _vp(self.features)), "features")
        self.force_simplex = self.force_simplex[:n]
        self.seed_values, self.seed_flags, self.features = self.seed_values[:n], self.seed_flags[:n], self.features[:n]
        # SKIP_SOLVE frame lists (None: the subset has none)
        has = np.zeros(max(n, 1), np.uint8)
        soff = np.zeros(n + 1, np.int32)
        sids = np.zeros(max(info.n_skip_solve_ids, 1), np.int32)
        abi.check(self.lib.dicegpu_subset_file_skip_solve(self.h, _vp(has), _vp(soff), _vp(sids)), "skip_solve")
        self.skip_solve = [list(sids[soff[i]:soff[i + 1]]) if has[i] else None for i in range(n)]

    def skip_solve_flags(self, frame):
        """Per-subset flags for dicegpu_set_skip_solve at frame id `frame`
        (frame_should_be_skipped over each subset's SKIP_SOLVE list)."""
        out = np.zeros(len(self.skip_solve), np.uint8)
        for i, ids in enumerate(self.skip_solve):
            if ids is None:
                continue
            a = np.ascontiguousarray(ids, dtype=np.int32)
            out[i] = self.lib.dicegpu_skip_solve_frame(_vp(a) if len(a) else None, len(a), int(frame))
        return out

    def apply_grid(self, schema, width, height, step_size):
        """Schema::initialize with a region-of-interest file and a step size."""
        abi.check(self.lib.dicegpu_subset_file_apply_grid(self.h, schema.ctx, width, height, step_size),
                  "subset_file_apply_grid")
        n = ctypes.c_int()
        p = abi.Params()
        abi.check(self.lib.dicegpu_get_params(schema.ctx, ctypes.byref(p)), "get_params")
        self.lib.dicegpu_regular_grid(self.h, width, height, step_size, p.subset_size, None, None, None, 0,
                                      ctypes.byref(n))
        schema.n = n.value

    def apply(self, schema):
        abi.check(self.lib.dicegpu_subset_file_apply(self.h, schema.ctx), "subset_file_apply")
        schema.n = self.info.n_subsets

    def close(self):
        if getattr(self, "h", None):
            self.lib.dicegpu_subset_file_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def regular_grid(subset_file, width, height, step_size, subset_size):
    """create_regular_grid_of_correlation_points: (xy n x 2, neighbour ids,
    seed region per point) for a region-of-interest file (or None: the whole
    image), in the reference's order."""
    lib = abi.load_library()
    h = subset_file.h if subset_file is not None else None
    n = ctypes.c_int()
    rc = lib.dicegpu_regular_grid(h, width, height, step_size, subset_size, None, None, None, 0, ctypes.byref(n))
    if rc not in (0, abi.ERR_ARG) or (rc == abi.ERR_ARG and n.value == 0):
        raise SubsetFileError("regular grid: %s" % abi.ERR_NAMES.get(rc, rc))
    xy = np.zeros((max(n.value, 1), 2), np.float64)
    neigh = np.zeros(max(n.value, 1), np.int32)
    seed = np.zeros(max(n.value, 1), np.int32)
    abi.check(lib.dicegpu_regular_grid(h, width, height, step_size, subset_size, _vp(xy), _vp(neigh), _vp(seed),
                                       n.value, ctypes.byref(n)), "regular_grid")
    return xy[:n.value], neigh[:n.value], seed[:n.value]
