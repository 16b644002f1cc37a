/*
 * dicegpu.h -- C ABI of the B200 subset-correlation library (libdicegpu.so).
 *
 * This header is the drop-in boundary for DICe's local subset-correlation hot
 * path: warp of the subset pixels by the affine or quadratic shape function,
 * Keys-4 / bicubic / bilinear interpolation of the deformed image and its
 * gradients, the ZNSSD residual, the FP64 Gauss-Newton Hessian / right-hand
 * side / LU solve, and the Nelder-Mead simplex fallback, followed by the
 * per-subset epilogue (sigma, gamma, noise, contrast, active pixels, status).
 *
 * Every entry point returns int: 0 on success, a negative DICEGPU_ERR_* code
 * otherwise.  Nothing throws across this boundary.  Per-subset outcomes are
 * reported with the reference's Status_Flag integers (DICe.h:609-675).
 *
 * Reference interfaces replaced (paths inside the DICe project):
 *   Schema::execute_correlation()          src/core/DICe_Schema.cpp:1622-1792
 *   Schema::generic_correlation_routine()  src/core/DICe_Schema.cpp:2026-2368
 *   Objective_ZNSSD::computeUpdateFast()   src/core/DICe_Objective.cpp:430-657
 *   Objective::computeUpdateRobust()       src/core/DICe_Objective.cpp:369-388
 *   Objective::gamma() / sigma()           src/core/DICe_Objective.cpp:58-76, 150-184
 *   Subset::initialize() (DEF target)      src/base/DICe_Subset.cpp:373-440
 *   Image_::interpolate_*_all()            src/base/DICe_Image.cpp:394-425, 493-636, 834-883
 *   Image_::compute_gradients()            src/base/DICe_Image.cpp:1015-1093
 *   dice_correlate() (C API precedent)     src/api/DICe_api.h:129-133, DICe_api.cpp:51-151
 *
 * Field layout: per-subset state lives in a double array of stride
 * DICEGPU_FIELD_STRIDE, the analogue of the Schema's per-subset MultiField
 * values (double, DICe_Schema.h:543-551).  Column indices are DICEGPU_F_*.
 */
#ifndef DICEGPU_H
#define DICEGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DICEGPU_ABI_VERSION 1

/* ---- error codes (return values) ---------------------------------------- */
#define DICEGPU_OK              0
#define DICEGPU_ERR_ARG        -1   /* bad argument (dice_correlate returns -1 too, DICe_api.cpp:71-76) */
#define DICEGPU_ERR_CUDA       -2   /* a CUDA runtime call failed */
#define DICEGPU_ERR_STATE      -3   /* call order: e.g. no reference image yet */
#define DICEGPU_ERR_NOMEM      -4   /* device allocation failed */
#define DICEGPU_ERR_TIMEOUT    -5   /* a bounded device wait gave up (status word) */
#define DICEGPU_ERR_UNSUPPORTED -6  /* option outside the implemented path */
#define DICEGPU_ERR_DEVICE     -7   /* the device status word recorded an error */

/* ---- enums mirroring the reference (DICe.h) ------------------------------ */
/* Status_Flag, DICe.h:609-675 (only the values the path produces are named) */
#define DICEGPU_CORRELATION_SUCCESSFUL                 0
#define DICEGPU_INITIALIZE_USING_PREVIOUS_FRAME_SUCCESSFUL 1
#define DICEGPU_INITIALIZE_USING_NEIGHBOR_VALUE_SUCCESSFUL 3
#define DICEGPU_INITIALIZE_FAILED                      5
#define DICEGPU_CORRELATION_FAILED                     8
#define DICEGPU_SUBSET_CONSTRUCTION_FAILED             9
#define DICEGPU_LINEAR_SOLVE_FAILED                   10
#define DICEGPU_MAX_ITERATIONS_REACHED                11
#define DICEGPU_INITIALIZE_FAILED_BY_EXCEPTION        12
#define DICEGPU_JUMP_TOLERANCE_EXCEEDED               16
#define DICEGPU_HESSIAN_SINGULAR                      21
#define DICEGPU_FRAME_FAILED_DUE_TO_HIGH_GAMMA        23
#define DICEGPU_FRAME_FAILED_DUE_TO_NEGATIVE_SIGMA    24
#define DICEGPU_FRAME_SKIPPED                         30

/* Interpolation_Method, DICe.h:549-555 */
#define DICEGPU_BILINEAR    0
#define DICEGPU_BICUBIC     1
#define DICEGPU_KEYS_FOURTH 2

/* Optimization_Method, DICe.h:527-535 */
#define DICEGPU_SIMPLEX                     0
#define DICEGPU_GRADIENT_BASED              1
#define DICEGPU_SIMPLEX_THEN_GRADIENT_BASED 3
#define DICEGPU_GRADIENT_BASED_THEN_SIMPLEX 4

/* Shape_Function_Type, DICe.h:509-516 */
#define DICEGPU_AFFINE_SF    0
#define DICEGPU_QUADRATIC_SF 1

/* Gradient_Method, DICe.h:563-568 */
#define DICEGPU_FINITE_DIFFERENCE   0
#define DICEGPU_CONVOLUTION_5_POINT 1

/* ---- per-subset field columns (double) ----------------------------------- */
#define DICEGPU_FIELD_STRIDE   32
#define DICEGPU_F_COORD_X       0   /* SUBSET_COORDINATES_X_FS */
#define DICEGPU_F_COORD_Y       1   /* SUBSET_COORDINATES_Y_FS */
#define DICEGPU_F_DISP_X        2   /* SUBSET_DISPLACEMENT_X_FS */
#define DICEGPU_F_DISP_Y        3   /* SUBSET_DISPLACEMENT_Y_FS */
#define DICEGPU_F_ROT_Z         4   /* ROTATION_Z_FS */
#define DICEGPU_F_STRETCH_XX    5   /* NORMAL_STRETCH_XX_FS */
#define DICEGPU_F_STRETCH_YY    6   /* NORMAL_STRETCH_YY_FS */
#define DICEGPU_F_SHEAR_XY      7   /* SHEAR_STRETCH_XY_FS */
#define DICEGPU_F_QUAD_A        8   /* QUAD_A_FS .. QUAD_L_FS = 8..19 */
#define DICEGPU_F_SIGMA        20
#define DICEGPU_F_GAMMA        21
#define DICEGPU_F_BETA         22
#define DICEGPU_F_NOISE        23
#define DICEGPU_F_CONTRAST     24
#define DICEGPU_F_ACTIVE_PIXELS 25
#define DICEGPU_F_STATUS       26
#define DICEGPU_F_ITERATIONS   27
#define DICEGPU_F_MATCH        28
#define DICEGPU_F_CONDITION    29   /* CONDITION_NUMBER_FS (2x2 displacement block) */
#define DICEGPU_F_OMEGA        30

/* Uncertainty fields of Objective::computeUncertaintyFields
 * (DICe_Objective.cpp:193-299), written for a subset whenever its
 * Gauss-Newton solve converges (params.compute_uncertainty = 1), kept across
 * frames like the reference's mesh fields (zero until first written).  Rows
 * of DICEGPU_UNCERTAINTY_STRIDE doubles: FIELD_1 .. FIELD_7 (FIELD_8/9 need
 * an image deformer, which the local path has none of). */
#define DICEGPU_UNCERTAINTY_STRIDE 8
#define DICEGPU_U_COS_THETA_HAT    0   /* FIELD_1: cos angle(u_hat, grad phi) */
#define DICEGPU_U_COS_THETA        1   /* FIELD_2: 1 without an exact motion */
#define DICEGPU_U_ERROR_L2         2   /* FIELD_3 */
#define DICEGPU_U_RESIDUAL_ERROR   3   /* FIELD_4 */
#define DICEGPU_U_ERROR_GRAD_PHI   4   /* FIELD_5 */
#define DICEGPU_U_RESIDUAL         5   /* FIELD_6 */
#define DICEGPU_U_SSSIG            6   /* FIELD_7: mean squared gradient */

/* VSG strain rows (dicegpu_vsg_strain), DICEGPU_VSG_STRIDE doubles: the
 * VSG_Strain_Post_Processor fields (DICe_PostProcessor.h:105-117) and the
 * number of valid neighbours used. */
#define DICEGPU_VSG_STRIDE     8
#define DICEGPU_VSG_STRAIN_XX  0   /* Green-Lagrange strains */
#define DICEGPU_VSG_STRAIN_YY  1
#define DICEGPU_VSG_STRAIN_XY  2
#define DICEGPU_VSG_DUDX       3
#define DICEGPU_VSG_DUDY       4
#define DICEGPU_VSG_DVDX       5
#define DICEGPU_VSG_DVDY       6
#define DICEGPU_VSG_NEIGHBORS  7

/* dice_correlate's record, DICe_api.h:65: x, y, u, v, theta, sigma, gamma, beta, flag */
#define DICEGPU_API_STRIDE 9

/* ---- correlation parameters (POD stand-in for Teuchos::ParameterList) -----
 * Defaults (dicegpu_default_params) are dice_default_params,
 * src/core/DICe_ParameterUtilities.cpp:363-421. */
typedef struct dicegpu_params {
  int32_t shape_function;          /* DICEGPU_AFFINE_SF | DICEGPU_QUADRATIC_SF */
  int32_t enable_translation;      /* must be 1 (DICe_LocalShapeFunction.cpp:164) */
  int32_t enable_rotation;
  int32_t enable_normal_strain;
  int32_t enable_shear_strain;
  int32_t interpolation;           /* DICEGPU_BILINEAR | BICUBIC | KEYS_FOURTH */
  int32_t optimization;            /* DICEGPU_SIMPLEX ... GRADIENT_BASED_THEN_SIMPLEX */
  int32_t gradient_method;         /* DICEGPU_FINITE_DIFFERENCE | CONVOLUTION_5_POINT */
  int32_t max_solver_iterations_fast;    /* 25 */
  int32_t max_solver_iterations_robust;  /* 1000 */
  double  fast_solver_tolerance;         /* 1e-4 */
  double  robust_solver_tolerance;       /* 1e-6 */
  double  skip_solve_gamma_threshold;    /* 1e-10 */
  double  robust_delta_disp;             /* 1.0 */
  double  robust_delta_theta;            /* 0.1 */
  double  disp_jump_tol;                 /* 1e4 */
  double  theta_jump_tol;                /* 100 */
  double  levenberg_marquardt_regularization_factor; /* -1 (off unless > 0) */
  double  momentum_factor;               /* 0 (off unless != 0) */
  double  initial_gamma_threshold;       /* -1 (off) */
  double  final_gamma_threshold;         /* -1 (off) */
  int32_t normalize_gamma_with_active_pixels; /* 0 */
  int32_t output_beta;                   /* 0 */
  /* 1: deformed-image gradients are computed and interpolated (images fed as
   * arrays: Schema::set_def_image(w,h,array), DICe_Schema.cpp:339, so
   * use_ref_grads=false).  0: the reference-image gradients at the reference
   * pixel are used, rotated by theta (images fed from files,
   * DICe_Schema.cpp:185; DICe_LocalShapeFunction.cpp:375-376). */
  int32_t use_def_gradients;
  int32_t subset_size;                   /* square subsets: side length (odd) */
  /* Gaussian pre-filter of both images before their gradients
   * (gauss_filter_images, gauss_filter_mask_size: 5, 7, 9, 11 or 13;
   * Image_::post_allocation_tasks, DICe_Image.cpp:300-318). */
  int32_t gauss_filter_images;
  int32_t gauss_filter_mask_size;
  /* 1: converged Gauss-Newton solves also write the uncertainty fields
   * (DICEGPU_UNCERTAINTY_STRIDE rows, dicegpu_get_uncertainty); the
   * reference always computes them, the default here is 0 (off). */
  int32_t compute_uncertainty;
  /* Correlation_Routine (DICe.h:587-591): GENERIC_ROUTINE runs the subsets
   * independently; TRACKING_ROUTINE runs them in index order and, before
   * each subset with blocking subsets, deactivates the pixels its blockers
   * cover at their current parameters (Schema::execute_correlation,
   * DICe_Schema.cpp:1732-1762, check_for_blocking_subsets, :4529-4557). */
  int32_t correlation_routine;
  /* obstruction_skin_factor: stretch of a blocking subset's deformed
   * boundary about its vertex centroid (1.0; tracking defaults 1.8). */
  double  obstruction_skin_factor;
  /* override_force_simplex: 0 forces the simplex on subsets that block or
   * are blocked (DICe_Schema.cpp:2160-2185); 1 leaves them to
   * params.optimization. */
  int32_t override_force_simplex;
  /* use_subset_evolution (0; tracking defaults 1): in the tracking routine,
   * from the third frame of a sequence on, after a successful solve, a
   * conformal subset's excluded pixels that are visible at the solved
   * parameters take their deformed intensity as reference and join the
   * subset for the rest of the sequence
   * (Subset::turn_on_previously_obstructed_pixels, DICe_Subset.cpp:506-520;
   * DICe_Schema.cpp:2354-2360; the generic routine rebuilds its objectives
   * every frame, so evolution has no lasting effect there).  Excluded pixels
   * then stay in the subsets' pixel lists as inactive.  Set it, and the
   * routine, before dicegpu_set_subset_shapes; the state restarts with each
   * sequence (frame index 0). */
  int32_t use_subset_evolution;
  /* use_incremental_formulation (0): each frame after the first of a
   * sequence correlates against the previous frame's deformed image
   * (dicegpu_set_ref_from_def before the new deformed image, as DICe's main
   * sets the reference to prev_img(), DICe_Main.cpp:326-328); the subsets'
   * DISPLACEMENT_X / _Y start the frame at 0 and end it as the accumulated
   * displacement (DICe_Schema.cpp:1671-1675, 1775-1789); the other
   * parameters carry over.  The tracking routine re-reads the reference
   * intensities from the new reference (:1757-1759), evolved pixels
   * included. */
  int32_t use_incremental_formulation;
  /* initialization_method (DICEGPU_USE_FIELD_VALUES): where a subset's
   * initial guess comes from (Field_Value_Initializer::initial_guess,
   * DICe_Initializer.cpp:398-436).  USE_NEIGHBOR_VALUES takes the field
   * values of the subset's neighbour (dicegpu_set_neighbors; -1 or itself:
   * its own), every frame; USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY at the first
   * frame of a sequence only.  Subsets run in index order as in the
   * reference, so a neighbour with a lower index contributes this frame's
   * solution and one with a higher index its frame-start values; the device
   * runs the subsets in dependency waves (a chain of single subsets as one
   * sequential launch).  Other methods: DICEGPU_ERR_UNSUPPORTED. */
  int32_t initialization_method;
  /* skip_all_solves (0): every subset is only initialised, as for a subset
   * whose solve is skipped (dicegpu_set_skip_solve): sigma, gamma (and beta)
   * at its initial guess, STATUS_FLAG = FRAME_SKIPPED, ITERATIONS = -1
   * (Schema::generic_correlation_routine, DICe_Schema.cpp:2118-2143). */
  int32_t skip_all_solves;
} dicegpu_params;

/* Initialization_Method (DICe.h:473-489) */
#define DICEGPU_USE_FIELD_VALUES                    0
#define DICEGPU_USE_NEIGHBOR_VALUES                 1
#define DICEGPU_USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY 2

/* Correlation_Routine */
#define DICEGPU_GENERIC_ROUTINE  0
#define DICEGPU_TRACKING_ROUTINE 1

/* Fills *p with the reference defaults. Replaces dice_default_params. */
int dicegpu_default_params(dicegpu_params* p);
/* Fills *p with the reference's tracking defaults (tracking_default_params,
 * DICe_ParameterUtilities.cpp:297-345; use_tracking_default_params),
 * subset evolution included. */
int dicegpu_tracking_default_params(dicegpu_params* p);

/* Number of shape-function parameters N for these params (2..6 affine, 12 quadratic). */
int dicegpu_num_params(const dicegpu_params* p);

/* ---- context -------------------------------------------------------------- */
typedef struct dicegpu_ctx dicegpu_ctx;

/* Creates a context on the current CUDA device.  The context owns the device
 * images, gradients, subset tables and per-subset field buffers.  One context
 * per host thread; calls on one context are serialised on its stream.
 * Replaces the Schema constructor's role for the hot path (DICe_Schema.cpp:101-139). */
int dicegpu_create(const dicegpu_params* params, dicegpu_ctx** out);
int dicegpu_destroy(dicegpu_ctx* ctx);
int dicegpu_set_params(dicegpu_ctx* ctx, const dicegpu_params* params);
int dicegpu_get_params(dicegpu_ctx* ctx, dicegpu_params* params);
/* The stream every later call on ctx is issued on (a cudaStream_t; NULL = legacy default). */
int dicegpu_set_stream(dicegpu_ctx* ctx, void* stream);

/* Images are row-major float [h][w].  `on_device` = 1 when `pixels` is a device
 * pointer (copied device to device), 0 for host memory.  The reference image
 * gets finite-difference gradients (Image_::compute_gradients,
 * DICe_Image.cpp:1015-1093); the deformed image gets them when
 * params.use_def_gradients is 1.  Replaces Schema::set_ref_image /
 * set_def_image(w,h,array) (DICe_Schema.cpp:328-349). */
int dicegpu_set_ref_image(dicegpu_ctx* ctx, int w, int h, const float* pixels, int on_device);
int dicegpu_set_def_image(dicegpu_ctx* ctx, int w, int h, const float* pixels, int on_device);

/* The same with 8- or 16-bit pixels (host or device memory), converted to
 * float of the same value on the device, as the reference's image readers
 * store them (DICe_ImageIO.cpp:480-490); the raw bytes cross PCIe, not the
 * floats.  pixel_type: DICEGPU_PIXEL_U8, DICEGPU_PIXEL_U16 or
 * DICEGPU_PIXEL_F32.  The optional Gaussian filter and the gradients follow
 * as for float images. */
#define DICEGPU_PIXEL_F32 0
#define DICEGPU_PIXEL_U8  1
#define DICEGPU_PIXEL_U16 2
int dicegpu_set_ref_image_typed(dicegpu_ctx* ctx, int w, int h, const void* pixels, int pixel_type,
                                int on_device);
int dicegpu_set_def_image_typed(dicegpu_ctx* ctx, int w, int h, const void* pixels, int pixel_type,
                                int on_device);

/* Square subsets of params.subset_size centred on the COORD_X/COORD_Y field
 * columns (Subset(cx,cy,w,h), DICe_Subset.cpp:78-113).  `fields` is a host
 * array of n * DICEGPU_FIELD_STRIDE doubles: coordinates plus the initial
 * shape-function fields (zeros for affine; QUAD_A = QUAD_H = 1 for quadratic,
 * as Quadratic_Shape_Function::reset_fields).  SIGMA = -1 marks a subset whose
 * initializer fails (DICe_Initializer.cpp:415-435). */
int dicegpu_set_subsets(dicegpu_ctx* ctx, int n, const double* fields);

/* Arbitrary-shape subsets (coordinate-array Subset ctor, DICe_Subset.cpp:49-76):
 * subset i owns pixels [offsets[i], offsets[i+1]) of px/py (global pixel
 * coordinates, row-major order).  Replaces params.subset_size for these subsets. */
int dicegpu_set_subset_pixels(dicegpu_ctx* ctx, int n, const int32_t* offsets,
                              const int32_t* px, const int32_t* py);

/* Conformal subsets built on the device from shapes (Subset(cx, cy,
 * Conformal_Area_Def), DICe_Subset.cpp:115-168, with Circle / Rectangle /
 * Polygon::get_owned_pixels, DICe_Shape.cpp:136-420): each subset's pixels
 * are the union of its boundary shapes (role 0), ordered by (y, x), minus
 * the pixels inside its excluded shapes (role 1, tested at the clamped
 * coordinates as deactivate_pixels does).  The reference keeps excluded
 * pixels in the list as inactive; here they are dropped, which gives the same
 * results except for the uncertainty fields' pixel count.  Negative
 * coordinates are clamped to 0 as the reference's constructor does.  A
 * subset without boundary shapes is a square of params.subset_size (as a
 * subset-file subset without a conformal definition is), empty when that is
 * below 1.  Obstructed shapes (role 2) are static regions of the image: a
 * subset pixel whose deformed position rounds into one is deactivated for
 * that evaluation (Subset::is_obstructed_pixel, DICe_Subset.cpp:446-460,
 * tested in Subset::initialize, :412-415).
 * Polygons use the reference's winding-angle test (float atan2 sums against
 * pi) with atan2 correctly rounded to float: a pixel lying exactly on an edge
 * is decided by the last bit of atan2f, which varies between CPU math
 * libraries; correct rounding makes that choice portable.  The
 * subsets must already exist (dicegpu_set_subsets); shapes and vertices are
 * host arrays.  Replaces the host-side construction of pixel lists
 * (dicegpu_set_subset_pixels). */
#define DICEGPU_SHAPE_CIRCLE    0
#define DICEGPU_SHAPE_RECTANGLE 1
#define DICEGPU_SHAPE_POLYGON   2
#define DICEGPU_ROLE_BOUNDARY   0
#define DICEGPU_ROLE_EXCLUDED   1
#define DICEGPU_ROLE_OBSTRUCTED 2
typedef struct dicegpu_shape {
  int32_t kind;            /* DICEGPU_SHAPE_* */
  int32_t subset;          /* owning subset index */
  int32_t role;            /* DICEGPU_ROLE_* */
  int32_t cx, cy;          /* circle / rectangle centroid */
  int32_t width, height;   /* rectangle */
  float radius;            /* circle */
  int32_t vertex_offset, vertex_count;   /* polygon: into vx / vy */
} dicegpu_shape;
int dicegpu_set_subset_shapes(dicegpu_ctx* ctx, int n_shapes, const dicegpu_shape* shapes,
                              const int32_t* vx, const int32_t* vy);

/* Blocking subsets (BLOCKING_SUBSETS of a conformal subset definition,
 * Schema::obstructing_subset_ids_): subset i is blocked by ids[offsets[i] ..
 * offsets[i+1]).  Under DICEGPU_TRACKING_ROUTINE, before subset i runs, the
 * pixels covered by each conformal blocker's boundary (its polygons and
 * rectangles mapped by the blocker's parameters, rounded, and stretched by
 * params.obstruction_skin_factor about their vertex centroid: get_owned_pixels
 * with a shape function, DICe_Shape.cpp:136-219, 322-396) are deactivated
 * in subset i.  A blocker earlier in index order contributes its parameters
 * of this frame, a later one those it had when the frame started.  Square
 * blockers cover nothing (Subset::deformed_shapes, DICe_Subset.cpp:462-476);
 * a blocker with a circular boundary is DICEGPU_ERR_UNSUPPORTED (the
 * reference throws there).  Blocked and blocking subsets use the simplex
 * unless params.override_force_simplex.  offsets == NULL clears the lists.
 * Call after dicegpu_set_subset_shapes. */
int dicegpu_set_blocking(dicegpu_ctx* ctx, const int32_t* offsets, const int32_t* ids);

/* VSG_Strain_Post_Processor::execute (DICe_PostProcessor.cpp:931-1130) on
 * the context's field rows: each subset's neighbours within window_size / 2
 * pixels (strain_window_size_in_pixels; the reference's kd-tree radius
 * search, squared distance in float < r^2 + 1e-5) with sigma >= 0 fit u and v
 * by planes in double, giving du/dx .. dv/dy and the Green-Lagrange strains.
 * Fewer than three valid neighbours, an invalid subset, or a reciprocal
 * condition number below 1e-12 give zeros and set the subset's MATCH field
 * to -1, as the reference does.  The reference estimates the condition
 * number (GECON); it is computed exactly here, which differs only for
 * nearly collinear neighbourhoods.  Writes n rows of DICEGPU_VSG_STRIDE
 * doubles to out (device memory when on_device, else host; NULL: kept on the
 * device only).  window_size < 0: the -window_size nearest subsets, valid or
 * not, form the neighbourhood (the reference's knnSearch,
 * DICe_PostProcessor.cpp:185-205) and the nearest (the subset itself) must
 * be valid; distances are the float squared distances, ties broken by
 * subset index where the reference's kd-tree breaks them by its traversal
 * order, so the two can differ only when several subsets tie at the k-th
 * distance.  -window_size larger than the subset count is DICEGPU_ERR_ARG. */
int dicegpu_vsg_strain(dicegpu_ctx* ctx, int window_size, double* out, int on_device);

/* Copies the context's subset pixel lists to host memory: offsets[n + 1]
 * and, when px / py are not NULL, offsets[n] coordinates each. */
int dicegpu_get_subset_pixels(dicegpu_ctx* ctx, int32_t* offsets, int32_t* px, int32_t* py);
/* NEIGHBOR_ID per subset (the decomposition's neighbor_ids, e.g. the
 * regular grid's snake predecessor); NULL clears them (every subset its own
 * neighbour).  Ids outside [0, n) count as -1. */
int dicegpu_set_neighbors(dicegpu_ctx* ctx, const int32_t* neighbor_ids);
/* Schema::post_execution_tasks + set_ref_image(prev_img()) of an
 * incremental sequence: the current deformed image (filtered, if the
 * params filter) becomes the reference and its gradients are computed;
 * device copies only, so it can be captured with a sequence. */
int dicegpu_set_ref_from_def(dicegpu_ctx* ctx);
/* Per-subset "skip the solve" flags for the following frames (n bytes,
 * non-zero: skip; NULL clears them): a skipped subset is initialised from
 * its field values as usual, then only evaluated there -- sigma, gamma,
 * beta, contrast, active pixels -- and recorded with STATUS_FLAG =
 * FRAME_SKIPPED and ITERATIONS = -1, without the jump or gamma tests
 * (DICe_Schema.cpp:2051-2059, 2118-2143; SKIP_SOLVE in a subset file).
 * dicegpu_skip_solve_frame gives a subset's flag for a frame from its
 * SKIP_SOLVE frame list. */
int dicegpu_set_skip_solve(dicegpu_ctx* ctx, int n, const uint8_t* flags);
/* frame_should_be_skipped (DICe_Schema.cpp:4945-4960): with the ascending
 * frame ids of a SKIP_SOLVE list (count 0: always skip), 1 when the solve
 * of frame `frame` is skipped -- frame ids toggle solving off and on,
 * starting on. */
int dicegpu_skip_solve_frame(const int32_t* frame_ids, int count, int frame);

/* Subset evolution state of the list pixels (use_subset_evolution in the
 * tracking routine, with conformal subsets that have excluded shapes):
 * state[offsets[n]] 0 inactive (excluded and not yet seen), 1 active, 2
 * turned on (Subset::turn_on_previously_obstructed_pixels), and
 * ref_values[offsets[n]] the reference intensities the turned-on pixels took
 * (Subset::ref_intensities_).  Either pointer may be NULL.  DICEGPU_ERR_STATE
 * when the lists carry no evolution state. */
int dicegpu_get_subset_pixel_state(dicegpu_ctx* ctx, uint8_t* state, float* ref_values);
/* Per-subset FORCE_SIMPLEX flags (DICe_Schema.cpp:2162-2165); NULL clears them. */
int dicegpu_set_force_simplex(dicegpu_ctx* ctx, int n, const uint8_t* flags);

/* Copies the n * DICEGPU_FIELD_STRIDE field array back to host memory
 * (waits for the context's stream). */
int dicegpu_get_fields(dicegpu_ctx* ctx, double* fields_out);
/* Copies the n * DICEGPU_UNCERTAINTY_STRIDE uncertainty fields to host
 * memory (FIELD_1..FIELD_7 of Objective::computeUncertaintyFields,
 * DICe_Objective.cpp:193-299).  DICEGPU_ERR_STATE unless
 * params.compute_uncertainty is set. */
int dicegpu_get_uncertainty(dicegpu_ctx* ctx, double* out);

/* Number of subsets of the context (0 before dicegpu_set_subsets). */
int dicegpu_num_subsets(dicegpu_ctx* ctx, int* n);

/* Device pointer of the field array (n * DICEGPU_FIELD_STRIDE doubles). */
int dicegpu_fields_device_ptr(dicegpu_ctx* ctx, double** dptr);
/* Asynchronous copies of the whole field array on the context's stream
 * (`on_device` = 1 for device memory, 0 for host memory; pinned host memory
 * keeps the copy asynchronous).  dicegpu_load_fields restarts the sequence:
 * the next frame is frame 0 again.  No synchronisation. */
int dicegpu_load_fields(dicegpu_ctx* ctx, const double* src, int on_device);
int dicegpu_store_fields(dicegpu_ctx* ctx, double* dst, int on_device);

/* One frame of local DIC over every subset: initial guess from the field
 * values (USE_FIELD_VALUES), Gauss-Newton and/or simplex per
 * params.optimization, jump / sigma / gamma tests, record_step.  Runs as one
 * persistent work-stealing launch.  The first call after dicegpu_set_subsets
 * is frame 0 (field-of-view check, DICe_Schema.cpp:2036-2048).
 * Replaces Schema::execute_correlation() (DICe_Schema.cpp:1622). */
int dicegpu_execute_correlation(dicegpu_ctx* ctx);

/* The same frame run as one kernel launch per subset (the plain, unbatched
 * GPU path the batched launch is compared with). */
int dicegpu_execute_correlation_plain(dicegpu_ctx* ctx);

/* Frame sequences as one CUDA graph.  dicegpu_capture_sequence records, for
 * frames k = 0..n-1, the device-to-device copy of frames[k] (device pointers
 * to w x h float images of the reference's size), its gradients, and one
 * frame of correlation initialised from the previous frame; when
 * `reset_fields` (device pointer, n_subsets * DICEGPU_FIELD_STRIDE doubles)
 * is not NULL the graph first reloads the fields from it and its first frame
 * is frame 0.  dicegpu_launch_sequence replays the graph on the context's
 * stream.  The frame pointers and the field source are read at every replay,
 * so their contents may change between replays.  Replaces the host loop of
 * set_def_image + execute_correlation (DICe_Main.cpp:324-357). */
int dicegpu_capture_sequence(dicegpu_ctx* ctx, int n, const float* const* frames,
                             const double* reset_fields);
int dicegpu_launch_sequence(dicegpu_ctx* ctx);

/* Chooses the persistent kernel's launch shape for the current images,
 * subsets and parameters: times one frame for each candidate (warps per CTA
 * x CTAs per SM), restoring the fields after each trial, keeps the fastest
 * and caches it per (device, shape function, interpolation, subset size) for
 * later contexts.  The result is applied to the context and returned. */
int dicegpu_autotune(dicegpu_ctx* ctx, int* warps_per_cta, int* ctas_per_sm, float* best_ms);

/* Number of kernel launches this context issued since creation. */
int dicegpu_launch_count(dicegpu_ctx* ctx, int64_t* count);

/* Launch shape of the persistent kernel: warps per CTA (one CTA solves one
 * subset at a time; 1-8, default 4) and CTAs per SM (0: as many as fit); 0
 * keeps the current value.  Until a shape is set here or by
 * dicegpu_autotune, a launch with at most six subsets per default-shape CTA
 * (small tracking waves, small frames, per-subset launches) and a chain of
 * single-subset waves run on CTAs of eight warps. */
int dicegpu_set_launch_shape(dicegpu_ctx* ctx, int warps_per_cta, int ctas_per_sm);
int dicegpu_get_launch_shape(dicegpu_ctx* ctx, int* warps_per_cta, int* ctas_per_sm);

/* ---- stride-9 API (mirror of dice_correlate) ------------------------------
 * Replaces dice_correlate (DICe_api.cpp:51-151); update_params is its
 * `const bool update_params`.  points: n * 9 floats [x, y, u, v, theta,
 * sigma, gamma, beta, flag]; u, v, theta are the guess, and the results
 * overwrite columns 2..8.  Images are host float arrays of equal size.
 *
 * Like the reference's static Schema, one context persists across calls (on
 * the device current at the first call, which later calls must keep):
 *  - the first call creates it from params (NULL: the tracking defaults of
 *    dicegpu_tracking_default_params, as DICe_api.cpp:84-93), square subsets
 *    of subset_size at the points' coordinates, and ref_img;
 *  - every later call keeps that reference image, subset size and subset
 *    count (ref_img and subset_size are not read again; another n_points is
 *    rejected with DICEGPU_ERR_ARG), writes the nine columns of every subset
 *    over the context's field rows (the other columns carry over), correlates
 *    def_img as the next frame of the sequence, and re-reads params (NULL:
 *    the tracking defaults) only when update_params is non-zero;
 *  - dicegpu_correlate_reset releases the context; the next call starts a
 *    new one.  A call that fails after the checks below releases it too.
 * Calls are serialised by a lock.  Returns -1 on the reference's argument
 * checks (DICe_api.cpp:71-76: image sizes differ, subset_size < 1,
 * n_points < 1), DICEGPU_ERR_UNSUPPORTED for a shape function other than
 * affine (the reference throws, DICe_api.cpp:116). */
int dicegpu_correlate(float* points, int n_points, int subset_size,
                      const float* ref_img, int ref_w, int ref_h,
                      const float* def_img, int def_w, int def_h,
                      const dicegpu_params* params, int update_params);
int dicegpu_correlate_reset(void);

/* ---- per-call kernels for the Objective / Image interfaces --------------- */
/* Interpolates the context's deformed image (and its gradients when present)
 * at n points xy[2n] with `method`.  Device or host pointers per on_device.
 * Replaces Image_::interpolate_{bilinear,bicubic,keys_fourth}_all. */
int dicegpu_interpolate(dicegpu_ctx* ctx, int method, int n, const float* xy,
                        float* intensity, float* grad_x, float* grad_y, int on_device);

/* Finite-difference gradients of a float image (both device pointers).
 * Replaces Image_::compute_gradients (DICe_Image.cpp:1015-1093). */
int dicegpu_image_gradients(int w, int h, const float* d_img, float* d_gx, float* d_gy,
                            int method, void* stream);

/* Gaussian filter of a float image with a mask_size x mask_size mask (5, 7,
 * 9, 11 or 13); pixels closer than mask_size/2+1 to an edge keep their
 * value.  d_in and d_out are device pointers to different buffers.
 * Replaces Image_::gauss_filter (DICe_Image.cpp:1194-1230).  Images smaller
 * than the mask are rejected with DICEGPU_ERR_ARG, as the reference
 * throws. */
int dicegpu_gauss_filter(int w, int h, const float* d_in, float* d_out, int mask_size,
                         void* stream);

/* The same gradients as dicegpu_image_gradients, computed without allocating
 * any device memory.  No counterpart in the reference: it exists for callers
 * that cannot call cudaMalloc -- hosts that own all device memory through
 * their own pool or budget, and per-frame loops that cannot afford the
 * device-wide wait of cudaFree.  The smoothing step's two intermediate
 * planes live in a file-scope device array of 2 * DICEGPU_NOALLOC_MAX_PIXELS
 * floats (8 MiB) that every GPU loading the library holds until exit.
 * With DICEGPU_CONVOLUTION_5_POINT, images larger than
 * DICEGPU_NOALLOC_MAX_PIXELS pixels are rejected with DICEGPU_ERR_ARG;
 * DICEGPU_FINITE_DIFFERENCE uses no intermediate planes and takes any size.
 * The first 5-point call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and caches it per device for the process; the
 * cached address belongs to that device's context, so after a
 * cudaDeviceReset of that device it is stale and the 5-point method must not
 * be called on it again.  All calls share the one array: calls whose GPU
 * work overlaps (other streams, other host threads) race on it and must be
 * serialised by the caller.  Both image pointers are device memory. */
#define DICEGPU_NOALLOC_MAX_PIXELS (1024 * 1024)
int dicegpu_image_gradients_noalloc(int w, int h, const float* d_img, float* d_gx, float* d_gy,
                                    int method, void* stream);

/* Objective::gamma for every subset at the parameters in `fields` (host,
 * n * stride): writes gamma per subset to gamma_out (host). */
int dicegpu_gamma(dicegpu_ctx* ctx, const double* fields, double* gamma_out);

/* Objective_ZNSSD::computeUpdateFast (DICe_Objective.cpp:430-657) for every
 * subset on its own: a fresh subset, the shape function initialised from the
 * subset's row of `fields` (host, n * DICEGPU_FIELD_STRIDE), Gauss-Newton to
 * convergence.  The updated shape-function columns (and CONDITION) are
 * written back into `fields`; num_iterations and the Status_Flag
 * (CORRELATION_SUCCESSFUL, MAX_ITERATIONS_REACHED, HESSIAN_SINGULAR) per
 * subset go to the two host arrays of n entries.  With
 * params.compute_uncertainty a converged solve also writes the subset's
 * uncertainty row, as the reference does. */
int dicegpu_compute_update_fast(dicegpu_ctx* ctx, double* fields, int32_t* num_iterations,
                                int32_t* status);

/* Objective::computeUpdateRobust (DICe_Objective.cpp:369-388): the
 * Nelder-Mead simplex (Simplex::minimize, DICe_Simplex.cpp:60-277) for every
 * subset on its own, same in/out convention as dicegpu_compute_update_fast;
 * the shape function is left where the simplex leaves it. */
int dicegpu_compute_update_robust(dicegpu_ctx* ctx, double* fields, int32_t* num_iterations,
                                  int32_t* status);

/* Objective::sigma (DICe_Objective.cpp:150-184) for every subset at the
 * parameters of its row of `fields`, after the subset has been initialised on
 * the deformed image at those parameters (the state sigma reads in the
 * correlation routine).  sigma_out and noise_out (noise_std_dev; may be NULL)
 * are host arrays of n doubles. */
int dicegpu_sigma(dicegpu_ctx* ctx, const double* fields, double* sigma_out, double* noise_out);

/* Reverse-mode derivative of the subset objective (no counterpart in the
 * reference, which has no derivative code: it differentiates the forward map
 * the reference evaluates -- warp by the shape function, Keys fourth-order
 * interpolation of the deformed image, Objective::gamma over the active
 * pixels, DICe_Objective.cpp:58-76).  For every subset at the parameters of
 * its row of d_fields (device, n * DICEGPU_FIELD_STRIDE):
 *   objective 0: gamma;  objective 1: sum ((G - mean G) - (F - mean F))^2,
 *   whose derivative is twice the Gauss-Newton right-hand side q.
 *   grad_source 0: the exact derivative of the Keys interpolant;
 *   grad_source 1: the Keys interpolation of the gradient images (needs
 *   params.use_def_gradients), as the Gauss-Newton residuals use.
 * d_seed (n doubles, NULL: all ones) weights each subset's objective.
 * Outputs (device, each may be NULL): d_value n objective values (-1 where
 * the objective is undefined), d_dparams n * 12 derivatives in parameter-slot
 * order (affine: u, v, theta, ex, ey, gxy; quadratic: A..L), d_ddef the W * H
 * derivative with respect to the deformed image's intensities, ADDED to what
 * the buffer holds.  Keys interpolation only (DICEGPU_ERR_UNSUPPORTED
 * otherwise).  Asynchronous on the context's stream. */
int dicegpu_adjoint(dicegpu_ctx* ctx, const double* d_fields, const double* d_seed, int objective,
                    int grad_source, double* d_value, double* d_dparams, float* d_ddef);

/* Error word the device kernels write instead of trapping (0 = none). */
int dicegpu_device_status(dicegpu_ctx* ctx, int32_t* status);

/* Library version string. */
const char* dicegpu_version(void);

#ifdef __cplusplus
}
#endif
#endif /* DICEGPU_H */
