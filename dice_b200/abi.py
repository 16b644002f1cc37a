"""ctypes view of include/dicegpu.h: the parameter struct, field columns and
status codes, plus the loader of the in-tree libdicegpu.so.

The product is the C ABI in libdicegpu.so; this module only describes it to
Python callers (tests, bench.py).  Loading fails loudly when the library has
not been built: there is no CPU fallback.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libdicegpu.so")

# ---- enums (DICe.h) --------------------------------------------------------
CORRELATION_SUCCESSFUL = 0
INITIALIZE_USING_PREVIOUS_FRAME_SUCCESSFUL = 1
INITIALIZE_USING_NEIGHBOR_VALUE_SUCCESSFUL = 3
INITIALIZE_FAILED = 5
CORRELATION_FAILED = 8
SUBSET_CONSTRUCTION_FAILED = 9
LINEAR_SOLVE_FAILED = 10
MAX_ITERATIONS_REACHED = 11
INITIALIZE_FAILED_BY_EXCEPTION = 12
JUMP_TOLERANCE_EXCEEDED = 16
HESSIAN_SINGULAR = 21
FRAME_FAILED_DUE_TO_HIGH_GAMMA = 23
FRAME_FAILED_DUE_TO_NEGATIVE_SIGMA = 24
FRAME_SKIPPED = 30

BILINEAR, BICUBIC, KEYS_FOURTH = 0, 1, 2
SIMPLEX, GRADIENT_BASED, SIMPLEX_THEN_GRADIENT_BASED, GRADIENT_BASED_THEN_SIMPLEX = 0, 1, 3, 4
AFFINE_SF, QUADRATIC_SF = 0, 1
FINITE_DIFFERENCE, CONVOLUTION_5_POINT = 0, 1

# ---- field columns ----------------------------------------------------------
FIELD_STRIDE = 32
F_COORD_X, F_COORD_Y, F_DISP_X, F_DISP_Y, F_ROT_Z = 0, 1, 2, 3, 4
F_STRETCH_XX, F_STRETCH_YY, F_SHEAR_XY = 5, 6, 7
F_QUAD_A = 8
F_SIGMA, F_GAMMA, F_BETA, F_NOISE, F_CONTRAST = 20, 21, 22, 23, 24
F_ACTIVE_PIXELS, F_STATUS, F_ITERATIONS, F_MATCH, F_CONDITION, F_OMEGA = 25, 26, 27, 28, 29, 30
API_STRIDE = 9
PIXEL_F32, PIXEL_U8, PIXEL_U16 = 0, 1, 2
SHAPE_CIRCLE, SHAPE_RECTANGLE, SHAPE_POLYGON = 0, 1, 2
ROLE_BOUNDARY, ROLE_EXCLUDED, ROLE_OBSTRUCTED = 0, 1, 2
GENERIC_ROUTINE, TRACKING_ROUTINE = 0, 1
USE_FIELD_VALUES, USE_NEIGHBOR_VALUES, USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY = 0, 1, 2


class Shape(ctypes.Structure):
    """dicegpu_shape: one boundary (role 0) or excluded (role 1) shape of a
    conformal subset (Conformal_Area_Def, DICe_Shape.h)."""
    _fields_ = [("kind", ctypes.c_int32), ("subset", ctypes.c_int32), ("role", ctypes.c_int32),
                ("cx", ctypes.c_int32), ("cy", ctypes.c_int32), ("width", ctypes.c_int32),
                ("height", ctypes.c_int32), ("radius", ctypes.c_float), ("vertex_offset", ctypes.c_int32),
                ("vertex_count", ctypes.c_int32)]


def circle(subset, cx, cy, radius, role=0):
    return Shape(SHAPE_CIRCLE, subset, role, int(cx), int(cy), 0, 0, float(radius), 0, 0)


def rectangle(subset, cx, cy, width, height, role=0):
    return Shape(SHAPE_RECTANGLE, subset, role, int(cx), int(cy), int(width), int(height), 0.0, 0, 0)


def polygon(subset, vertex_offset, vertex_count, role=0):
    return Shape(SHAPE_POLYGON, subset, role, 0, 0, 0, 0, 0.0, int(vertex_offset), int(vertex_count))


def shape_array(shapes):
    return (Shape * len(shapes))(*shapes)
UNCERTAINTY_STRIDE = 8
VSG_STRIDE = 8
VSG_STRAIN_XX, VSG_STRAIN_YY, VSG_STRAIN_XY, VSG_DUDX, VSG_DUDY, VSG_DVDX, VSG_DVDY, VSG_NEIGHBORS = range(8)

ERR_NAMES = {0: "OK", -1: "ERR_ARG", -2: "ERR_CUDA", -3: "ERR_STATE", -4: "ERR_NOMEM",
             -5: "ERR_TIMEOUT", -6: "ERR_UNSUPPORTED", -7: "ERR_DEVICE"}
OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NOMEM, ERR_TIMEOUT, ERR_UNSUPPORTED, ERR_DEVICE = 0, -1, -2, -3, -4, -5, -6, -7


class Params(ctypes.Structure):
    """dicegpu_params (include/dicegpu.h)."""
    _fields_ = [
        ("shape_function", ctypes.c_int32),
        ("enable_translation", ctypes.c_int32),
        ("enable_rotation", ctypes.c_int32),
        ("enable_normal_strain", ctypes.c_int32),
        ("enable_shear_strain", ctypes.c_int32),
        ("interpolation", ctypes.c_int32),
        ("optimization", ctypes.c_int32),
        ("gradient_method", ctypes.c_int32),
        ("max_solver_iterations_fast", ctypes.c_int32),
        ("max_solver_iterations_robust", ctypes.c_int32),
        ("fast_solver_tolerance", ctypes.c_double),
        ("robust_solver_tolerance", ctypes.c_double),
        ("skip_solve_gamma_threshold", ctypes.c_double),
        ("robust_delta_disp", ctypes.c_double),
        ("robust_delta_theta", ctypes.c_double),
        ("disp_jump_tol", ctypes.c_double),
        ("theta_jump_tol", ctypes.c_double),
        ("levenberg_marquardt_regularization_factor", ctypes.c_double),
        ("momentum_factor", ctypes.c_double),
        ("initial_gamma_threshold", ctypes.c_double),
        ("final_gamma_threshold", ctypes.c_double),
        ("normalize_gamma_with_active_pixels", ctypes.c_int32),
        ("output_beta", ctypes.c_int32),
        ("use_def_gradients", ctypes.c_int32),
        ("subset_size", ctypes.c_int32),
        ("gauss_filter_images", ctypes.c_int32),
        ("gauss_filter_mask_size", ctypes.c_int32),
        ("compute_uncertainty", ctypes.c_int32),
        ("correlation_routine", ctypes.c_int32),
        ("obstruction_skin_factor", ctypes.c_double),
        ("override_force_simplex", ctypes.c_int32),
        ("use_subset_evolution", ctypes.c_int32),
        ("use_incremental_formulation", ctypes.c_int32),
        ("initialization_method", ctypes.c_int32),
        ("skip_all_solves", ctypes.c_int32),
    ]

    def copy(self):
        p = Params()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(Params))
        return p


def default_params(**overrides):
    """dice_default_params (DICe_ParameterUtilities.cpp:363-421) with overrides."""
    p = Params()
    p.shape_function = AFFINE_SF
    p.enable_translation = 1
    p.interpolation = KEYS_FOURTH
    p.optimization = GRADIENT_BASED_THEN_SIMPLEX
    p.gradient_method = FINITE_DIFFERENCE
    p.max_solver_iterations_fast = 25
    p.max_solver_iterations_robust = 1000
    p.fast_solver_tolerance = 1.0e-4
    p.robust_solver_tolerance = 1.0e-6
    p.skip_solve_gamma_threshold = 1.0e-10
    p.robust_delta_disp = 1.0
    p.robust_delta_theta = 0.1
    p.disp_jump_tol = 10000.0
    p.theta_jump_tol = 100.0
    p.levenberg_marquardt_regularization_factor = -1.0
    p.momentum_factor = 0.0
    p.initial_gamma_threshold = -1.0
    p.final_gamma_threshold = -1.0
    p.use_def_gradients = 1
    p.subset_size = 21
    p.gauss_filter_images = 0
    p.gauss_filter_mask_size = 7
    p.correlation_routine = GENERIC_ROUTINE
    p.obstruction_skin_factor = 1.0
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def tracking_default_params(**overrides):
    """tracking_default_params (DICe_ParameterUtilities.cpp:297-345) with overrides."""
    p = default_params()
    p.correlation_routine = TRACKING_ROUTINE
    p.optimization = SIMPLEX
    p.enable_rotation = 1
    p.disp_jump_tol = 8.0
    p.theta_jump_tol = 0.1
    p.obstruction_skin_factor = 1.8
    p.override_force_simplex = 1
    p.use_subset_evolution = 1
    for k, v in overrides.items():
        if not hasattr(p, k):
            raise AttributeError(k)
        setattr(p, k, v)
    return p


def num_params(p):
    if p.shape_function == QUADRATIC_SF:
        return 12
    return 2 + (1 if p.enable_rotation else 0) + (2 if p.enable_normal_strain else 0) + \
        (1 if p.enable_shear_strain else 0)


_lib = None


def load_library(path=None):
    """Loads libdicegpu.so (built in-tree by dice_b200/csrc/Makefile)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError("libdicegpu.so is not built (%s); run __graft_entry__.build()" % path)
    lib = ctypes.CDLL(path)
    _declare(lib)
    if path == LIB_PATH:
        _lib = lib
    return lib


def _declare(lib):
    c_int, c_void_p, c_double_p = ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
    P = ctypes.POINTER(Params)
    sigs = {
        "dicegpu_default_params": (c_int, [P]),
        "dicegpu_num_params": (c_int, [P]),
        "dicegpu_create": (c_int, [P, ctypes.POINTER(c_void_p)]),
        "dicegpu_destroy": (c_int, [c_void_p]),
        "dicegpu_set_params": (c_int, [c_void_p, P]),
        "dicegpu_set_stream": (c_int, [c_void_p, c_void_p]),
        "dicegpu_set_ref_image": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int]),
        "dicegpu_set_def_image": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int]),
        "dicegpu_set_ref_image_typed": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_int]),
        "dicegpu_set_def_image_typed": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_int]),
        "dicegpu_set_subsets": (c_int, [c_void_p, c_int, c_void_p]),
        "dicegpu_set_subset_pixels": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
        "dicegpu_set_subset_shapes": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
        "dicegpu_get_subset_pixels": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "dicegpu_get_subset_pixel_state": (c_int, [c_void_p, c_void_p, c_void_p]),
        "dicegpu_set_ref_from_def": (c_int, [c_void_p]),
        "dicegpu_set_neighbors": (c_int, [c_void_p, c_void_p]),
        "dicegpu_set_blocking": (c_int, [c_void_p, c_void_p, c_void_p]),
        "dicegpu_get_params": (c_int, [c_void_p, P]),
        "dicegpu_subset_file_read": (c_int, [ctypes.c_char_p, c_int, c_int, ctypes.POINTER(c_void_p),
                                             ctypes.c_char_p, c_int]),
        "dicegpu_subset_file_parse": (c_int, [ctypes.c_char_p, ctypes.c_size_t, c_int, c_int,
                                              ctypes.POINTER(c_void_p), ctypes.c_char_p, c_int]),
        "dicegpu_subset_file_free": (c_int, [c_void_p]),
        "dicegpu_subset_file_get_info": (c_int, [c_void_p, c_void_p]),
        "dicegpu_subset_file_coordinates": (c_int, [c_void_p, c_void_p]),
        "dicegpu_subset_file_shapes": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "dicegpu_subset_file_blocking": (c_int, [c_void_p, c_void_p, c_void_p]),
        "dicegpu_subset_file_force_simplex": (c_int, [c_void_p, c_void_p]),
        "dicegpu_subset_file_seeds": (c_int, [c_void_p, c_void_p, c_void_p]),
        "dicegpu_subset_file_features": (c_int, [c_void_p, c_void_p]),
        "dicegpu_subset_file_skip_solve": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "dicegpu_subset_file_apply": (c_int, [c_void_p, c_void_p]),
        "dicegpu_output_create": (c_int, [P, ctypes.c_char_p, ctypes.c_char_p, c_int, c_void_p,
                                          ctypes.POINTER(c_void_p)]),
        "dicegpu_output_destroy": (c_int, [c_void_p]),
        "dicegpu_output_set_images": (c_int, [c_void_p, ctypes.c_char_p, ctypes.c_char_p]),
        "dicegpu_output_num_fields": (c_int, [c_void_p, ctypes.POINTER(c_int)]),
        "dicegpu_output_info_text": (c_int, [c_void_p, ctypes.c_char_p, ctypes.c_size_t,
                                             ctypes.POINTER(ctypes.c_size_t)]),
        "dicegpu_output_header_text": (c_int, [c_void_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t,
                                               ctypes.POINTER(ctypes.c_size_t)]),
        "dicegpu_output_row_text": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_void_p, ctypes.c_char_p,
                                            ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)]),
        "dicegpu_output_write_frame": (c_int, [c_void_p, ctypes.c_char_p, ctypes.c_char_p, c_int, c_int, c_int,
                                               c_int, c_void_p, c_void_p, c_void_p, c_int]),
        "dicegpu_vsg_strain": (c_int, [c_void_p, c_int, c_void_p, c_int]),
        "dicegpu_regular_grid": (c_int, [c_void_p, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                         c_int, ctypes.POINTER(c_int)]),
        "dicegpu_subset_file_apply_grid": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int]),
        "dicegpu_diff_files": (c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_double, ctypes.c_double, c_int,
                                       c_int, c_int, ctypes.POINTER(c_int), ctypes.c_char_p, ctypes.c_size_t]),
        "dicegpu_diff_text": (c_int, [ctypes.c_char_p, ctypes.c_size_t, ctypes.c_char_p, ctypes.c_size_t,
                                      ctypes.c_double, ctypes.c_double, c_int, c_int, ctypes.POINTER(c_int),
                                      ctypes.c_char_p, ctypes.c_size_t]),
        "dicegpu_tracking_default_params": (c_int, [P]),
        "dicegpu_set_force_simplex": (c_int, [c_void_p, c_int, c_void_p]),
        "dicegpu_get_fields": (c_int, [c_void_p, c_void_p]),
        "dicegpu_get_uncertainty": (c_int, [c_void_p, c_void_p]),
        "dicegpu_num_subsets": (c_int, [c_void_p, ctypes.POINTER(c_int)]),
        "dicegpu_compute_update_fast": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "dicegpu_compute_update_robust": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "dicegpu_sigma": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "dicegpu_adjoint": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p,
                                    c_void_p]),
        "dicegpu_fields_device_ptr": (c_int, [c_void_p, ctypes.POINTER(c_void_p)]),
        "dicegpu_load_fields": (c_int, [c_void_p, c_void_p, c_int]),
        "dicegpu_store_fields": (c_int, [c_void_p, c_void_p, c_int]),
        "dicegpu_execute_correlation": (c_int, [c_void_p]),
        "dicegpu_execute_correlation_plain": (c_int, [c_void_p]),
        "dicegpu_launch_count": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_int64)]),
        "dicegpu_capture_sequence": (c_int, [c_void_p, c_int, c_void_p, c_void_p]),
        "dicegpu_launch_sequence": (c_int, [c_void_p]),
        "dicegpu_autotune": (c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int),
                                     ctypes.POINTER(ctypes.c_float)]),
        "dicegpu_set_launch_shape": (c_int, [c_void_p, c_int, c_int]),
        "dicegpu_get_launch_shape": (c_int, [c_void_p, ctypes.POINTER(c_int), ctypes.POINTER(c_int)]),
        "dicegpu_correlate": (c_int, [c_void_p, c_int, c_int, c_void_p, c_int, c_int, c_void_p,
                                      c_int, c_int, P, c_int]),
        "dicegpu_correlate_reset": (c_int, []),
        "dicegpu_set_skip_solve": (c_int, [c_void_p, c_int, c_void_p]),
        "dicegpu_skip_solve_frame": (c_int, [c_void_p, c_int, c_int]),
        "dicegpu_interpolate": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_void_p,
                                        c_void_p, c_int]),
        "dicegpu_image_gradients": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                            c_void_p]),
        "dicegpu_gauss_filter": (c_int, [c_int, c_int, c_void_p, c_void_p, c_int, c_void_p]),
        "dicegpu_image_gradients_noalloc": (c_int, [c_int, c_int, c_void_p, c_void_p, c_void_p, c_int,
                                                    c_void_p]),
        "dicegpu_gamma": (c_int, [c_void_p, c_void_p, c_void_p]),
        "dicegpu_device_status": (c_int, [c_void_p, ctypes.POINTER(ctypes.c_int32)]),
        "dicegpu_version": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _ = c_double_p


def check(rc, what=""):
    if rc != 0:
        raise RuntimeError("%s failed: %s (%d)" % (what, ERR_NAMES.get(rc, "?"), rc))
    return rc
