/*
 * dice_oracle.h -- CPU oracle for the DICe local subset-correlation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a CPU restatement of the reference
 * algorithm (scalar_t = float, FP32 products, FP64 Hessian / RHS accumulation,
 * FP64 LU) used as the checker in tests/, in __graft_entry__.smoke() and as
 * the timed CPU baseline in bench.py.  The product path (libdicegpu.so) never
 * links, loads or calls it.
 *
 * Parity pin: tests/test_oracle_gold.py checks it against the reference's own
 * regression gold (tests/regression/parallel_subsets/gold/DICe_solution_0.txt,
 * tests/regression/single_speckled_shift/gold/) and the component
 * known-answer tests restated in tests/test_oracle_kat.py.
 *
 * Parameter, field and status conventions are those of include/dicegpu.h.
 */
#ifndef DICE_ORACLE_H
#define DICE_ORACLE_H

#include "dicegpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* One frame of Schema::execute_correlation over n subsets (GENERIC_ROUTINE,
 * USE_FIELD_VALUES).  Subsets are square (params->subset_size, centred on the
 * COORD fields) unless offsets/px/py give pixel lists.  `first_frame` enables
 * the frame-0 field-of-view test.  `nthreads` workers split the subsets in
 * contiguous ranges (the reference splits them over MPI ranks).  When
 * `oracle_gn_iters` is non-NULL it receives, per subset, the number of
 * Gauss-Newton iterations actually executed (for FLOP accounting).  When
 * `uncertainty` is non-NULL (n * DICEGPU_UNCERTAINTY_STRIDE doubles) every
 * converged Gauss-Newton solve writes its subset's uncertainty fields there,
 * as the reference always does. */
int oracle_execute_frame(const dicegpu_params* params, int w, int h,
                         const float* ref, const float* def, int n, double* fields,
                         const int32_t* offsets, const int32_t* px, const int32_t* py,
                         const uint8_t* force_simplex, int first_frame, int nthreads,
                         int32_t* gn_iters_out, int32_t* simplex_evals_out, double* uncertainty,
                         const int32_t* neighbors);

/* Image_::compute_gradients (finite difference, optional 5-point smoothing). */
int oracle_gradients(int w, int h, const float* img, int method, float* gx, float* gy);

/* Image_::gauss_filter with a mask_size x mask_size mask (5..13, odd). */
int oracle_gauss_filter(int w, int h, const float* in, float* out, int mask_size);

/* Image_::interpolate_*_all at n points (x,y interleaved). gx/gy may be NULL. */
int oracle_interpolate(int method, int w, int h, const float* img, const float* gx,
                       const float* gy, int n, const float* xy, float* out_i,
                       float* out_gx, float* out_gy);

/* The Gauss-Newton system (H: n x N x N, q: n x N) of computeUpdateFast at
 * the parameters of each (square) subset's field row, assembled once. */
int oracle_gn_system(const dicegpu_params* params, int w, int h, const float* ref,
                     const float* def, int n, const double* fields, double* H_out, double* q_out);

/* One Objective entry point per (square) subset at the parameters of its row
 * of `fields`: op 0 computeUpdateFast, 1 computeUpdateRobust, 2 sigma. */
int oracle_objective(const dicegpu_params* params, int w, int h, const float* ref,
                     const float* def, int n, double* fields, int op, int32_t* iters_out,
                     int32_t* status_out, double* sigma_out, double* noise_out);

/* Objective::gamma for each subset at the parameters in `fields`. */
int oracle_gamma(const dicegpu_params* params, int w, int h, const float* ref,
                 const float* def, int n, const double* fields, double* gamma_out);

/* Local_Shape_Function::map of n points (x,y interleaved) about (cx, cy) for
 * the parameters in the field row `fields` (DICEGPU_F_* columns). */
int oracle_map(const dicegpu_params* params, const double* fields, int n, const float* xy,
               float cx, float cy, float* out_xy);

/* Pixel lists of conformal subsets from shapes (get_owned_pixels); with
 * px == NULL only offsets[n + 1] is filled. */
int oracle_rasterize(int n, int n_shapes, const dicegpu_shape* shapes, const int32_t* vx,
                     const int32_t* vy, const double* fields, int square_size, int32_t* offsets,
                     int32_t* px, int32_t* py);

/* Schema::execute_correlation over subsets defined by shapes (boundary,
 * excluded, obstructed; squares where a subset has no boundary), with
 * blocking subsets (block_offsets[n+1], block_ids; NULL for none) under the
 * generic or tracking routine of params. */
int oracle_execute_frame_shapes(const dicegpu_params* params, int w, int h, const float* ref,
                                const float* def, int n, double* fields, int n_shapes,
                                const dicegpu_shape* shapes, const int32_t* vx, const int32_t* vy,
                                const int32_t* block_offsets, const int32_t* block_ids,
                                const uint8_t* force_simplex, int first_frame, int nthreads,
                                uint8_t* pix_flag, float* pix_f, int frame_index);

/* VSG_Strain_Post_Processor on n field rows (window > 0: radius window/2):
 * out n x 7 (strain xx, yy, xy, du/dx, du/dy, dv/dx, dv/dy), failed n flags. */
int oracle_vsg_strain(int n, const double* fields, int window, double* out, int32_t* failed);

/* Defaults of dice_default_params (same values as dicegpu_default_params). */
int oracle_default_params(dicegpu_params* p);

#ifdef __cplusplus
}
#endif
#endif
