/*
 * dicegpu_subset_file.h -- DICe subset files (host C++, in libdicegpu.so).
 *
 * Parses the subset-definition files a DICe input names as `subset_file`
 * and hands their subsets to a correlation context.  Replaces, for the local
 * correlation path (paths inside the DICe project):
 *   read_subset_file()   src/core/DICe_Parser.cpp:1098-1650
 *   read_shapes() / read_circle() / read_rectangle() / read_polygon()
 *                        src/core/DICe_Parser.cpp:1652-1860
 *   tokenize_line(), is_number()  src/core/DICe_Parser.cpp:1044-1096
 *   Schema::initialize(input_params, ...) with a subset file (coordinates,
 *   conformal definitions, blocking subsets, forced simplex, seeds)
 *                        src/core/DICe_Schema.cpp:1025-1145
 *
 * File format (keywords are case-insensitive, '#' starts a comment line):
 *   BEGIN SUBSET_COORDINATES  <x y per line>  END
 *   BEGIN CONFORMAL_SUBSET
 *     SUBSET_ID <id>
 *     BEGIN BOUNDARY | EXCLUDED | OBSTRUCTED
 *       BEGIN CIRCLE  CENTER <x y>  RADIUS <r>  END
 *       BEGIN RECTANGLE  CENTER <x y>  WIDTH <w>  HEIGHT <h>  END
 *         (or UPPER_LEFT <x y>  LOWER_RIGHT <x y>)
 *       BEGIN POLYGON  BEGIN VERTICES <x y per line> END  END
 *     END
 *     BEGIN BLOCKING_SUBSETS <id per line> END
 *     BEGIN SEED  DISPLACEMENT <u v>  [NORMAL_STRAIN <ex ey>]
 *                 [SHEAR_STRAIN <g>]  [ROTATION <t>]  END
 *     FORCE_SIMPLEX | USE_OPTICAL_FLOW | USE_PATH_FILE <f> | SKIP_SOLVE ...
 *     | TEST_FOR_MOTION | MOTION_WINDOW ...
 *   END
 *   BEGIN REGION_OF_INTEREST ... END   (a region with a seed; no coordinates)
 *
 * Errors: every entry point returns 0 or a negative DICEGPU_ERR_* code; a
 * file the reference rejects returns DICEGPU_ERR_ARG with the reason in `err`.
 */
#ifndef DICEGPU_SUBSET_FILE_H
#define DICEGPU_SUBSET_FILE_H

#include <stddef.h>
#include <stdint.h>

#include "dicegpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dicegpu_subset_file dicegpu_subset_file;

typedef struct dicegpu_subset_file_info {
  int32_t n_subsets;          /* coordinates read (0 for a region of interest) */
  int32_t n_shapes;           /* shapes of all conformal definitions */
  int32_t n_vertices;         /* polygon vertices of those shapes */
  int32_t n_blocking_ids;     /* entries of all BLOCKING_SUBSETS lists */
  int32_t n_conformal;        /* conformal definitions */
  int32_t region_of_interest; /* 1: a REGION_OF_INTEREST file */
  int32_t n_seeds;            /* definitions with a SEED */
  int32_t n_unsupported;      /* subsets using a feature listed under DICEGPU_SF_FEATURE_* */
  int32_t n_skip_solve_ids;   /* frame ids of all SKIP_SOLVE lists */
} dicegpu_subset_file_info;

/* Feature bits of dicegpu_subset_file_features: subset-file options that
 * select parts of the reference outside this library's correlation path
 * (other initializers, motion detection, a SKIP_SOLVE whose frame ids are in
 * another file).  A SKIP_SOLVE with its frame ids on the line is read:
 * dicegpu_subset_file_skip_solve. */
#define DICEGPU_SF_FEATURE_SKIP_SOLVE    1
#define DICEGPU_SF_FEATURE_OPTICAL_FLOW  2
#define DICEGPU_SF_FEATURE_PATH_FILE     4
#define DICEGPU_SF_FEATURE_MOTION_WINDOW 8
#define DICEGPU_SF_FEATURE_TEST_MOTION   16

/* Seed bits of dicegpu_subset_file_seeds */
#define DICEGPU_SF_SEED_DISPLACEMENT  1
#define DICEGPU_SF_SEED_NORMAL_STRAIN 2
#define DICEGPU_SF_SEED_SHEAR_STRAIN  4
#define DICEGPU_SF_SEED_ROTATION      8

/* Parses a subset file from a path or from memory.  width / height bound
 * the subset coordinates as the reference checks them (-1: unchecked).  On
 * failure *out is NULL and err (when err_len > 0) holds the reason. */
int dicegpu_subset_file_read(const char* path, int width, int height, dicegpu_subset_file** out, char* err,
                             int err_len);
int dicegpu_subset_file_parse(const char* text, size_t len, int width, int height, dicegpu_subset_file** out,
                              char* err, int err_len);
int dicegpu_subset_file_free(dicegpu_subset_file* f);

int dicegpu_subset_file_get_info(const dicegpu_subset_file* f, dicegpu_subset_file_info* info);
/* n_subsets (x, y) pairs, in file order: subset i is the i-th coordinate. */
int dicegpu_subset_file_coordinates(const dicegpu_subset_file* f, double* xy);
/* n_shapes shapes (subset = the definition's SUBSET_ID, role boundary /
 * excluded / obstructed) and n_vertices polygon vertices. */
int dicegpu_subset_file_shapes(const dicegpu_subset_file* f, dicegpu_shape* shapes, int32_t* vx, int32_t* vy);
/* Blocking lists per subset: offsets[n_subsets + 1], ids[n_blocking_ids]. */
int dicegpu_subset_file_blocking(const dicegpu_subset_file* f, int32_t* offsets, int32_t* ids);
/* FORCE_SIMPLEX per subset (n_subsets bytes). */
int dicegpu_subset_file_force_simplex(const dicegpu_subset_file* f, uint8_t* flags);
/* Seeds per subset: values[6 * i ..] = u, v, normal strain x, y, shear
 * strain, rotation; flags[i] = DICEGPU_SF_SEED_* bits present. */
int dicegpu_subset_file_seeds(const dicegpu_subset_file* f, double* values, uint8_t* flags);
/* SKIP_SOLVE per subset (DICe_Parser.cpp:1435-1463): has_skip[i] non-zero
 * when subset i has one; its ascending frame ids are frame_ids[offsets[i] ..
 * offsets[i + 1]) (offsets: n_subsets + 1 entries; frame_ids:
 * n_skip_solve_ids).  dicegpu_skip_solve_frame turns a list into the flag
 * of a frame for dicegpu_set_skip_solve. */
int dicegpu_subset_file_skip_solve(const dicegpu_subset_file* f, uint8_t* has_skip, int32_t* offsets,
                                   int32_t* frame_ids);
/* DICEGPU_SF_FEATURE_* bits per subset (n_subsets bytes). */
int dicegpu_subset_file_features(const dicegpu_subset_file* f, uint8_t* flags);

/* Schema::initialize with this subset file on a context whose params are
 * set: one subset per coordinate (field rows with the coordinates and the
 * seeds' values), the conformal definitions as shapes (subsets without one
 * are squares of params.subset_size), the blocking lists and the
 * FORCE_SIMPLEX flags.  DICEGPU_ERR_UNSUPPORTED for a region-of-interest
 * file (see dicegpu_subset_file_apply_grid) or a subset using a
 * DICEGPU_SF_FEATURE_* option; DICEGPU_ERR_ARG when
 * a subset is neither conformal nor given a size (params.subset_size < 1)
 * or a seed sets strains under the quadratic shape function (the reference
 * throws there). */
int dicegpu_subset_file_apply(const dicegpu_subset_file* f, dicegpu_ctx* ctx);

/* create_regular_grid_of_correlation_points (DICe_Decomp.cpp:868-1050):
 * subset centres every step_size pixels from subset_size - 1 in x and y,
 * kept when the centre lies in a region of interest (the REGION_OF_INTEREST
 * blocks of f in id order, or the whole image when f is NULL), no corner of
 * the subset lies in the region's excluded shapes, and the subset is at
 * least subset_size - 1 from the image's edges; in the reference's order:
 * each region's seed point (its SEED LOCATION rounded onto the grid, else
 * the first grid point), then a column-wise snake right of it, then one
 * left.  For each point: xy (2 doubles), neighbor_ids (the previous point
 * on its snake, the seed for a snake's first point when a seed was given,
 * else -1) and seed_roi (the region whose seed it is, else -1); any of them
 * may be NULL.  *n receives the number of points; DICEGPU_ERR_ARG when it
 * exceeds cap (nothing beyond cap is written) or a given seed is not a valid
 * point.  The reference's optional gradient threshold (sssig) is not
 * applied. */
int dicegpu_regular_grid(const dicegpu_subset_file* f, int width, int height, int step_size, int subset_size,
                         double* xy, int32_t* neighbor_ids, int32_t* seed_roi, int cap, int* n);

/* Schema::initialize with a region-of-interest file (or none: f NULL, the
 * whole image) and a step size: the grid's points become square subsets of
 * params.subset_size, the regions' seeds their field rows' initial values,
 * and the grid's neighbor_ids the subsets' neighbours
 * (dicegpu_set_neighbors). */
int dicegpu_subset_file_apply_grid(const dicegpu_subset_file* f, dicegpu_ctx* ctx, int width, int height,
                                   int step_size);

#ifdef __cplusplus
}
#endif

#endif /* DICEGPU_SUBSET_FILE_H */
