/*
 * dicegpu_results.h -- DICe text results: writer and comparator (host C++,
 * in libdicegpu.so).
 *
 * The writer produces the files Schema::write_output writes for the local
 * path (src/core/DICe_Schema.cpp:4327-4478) with Output_Spec's layout
 * (:4673-4943): the "***" information block, the header row, then one row
 * per subset or frame with every value printed "%4.4E" after rounding to
 * float (the reference prints a scalar_t).  The comparator is DICe_Diff
 * (tools/DICe_Diff.cpp): the same tokens, tolerance arithmetic, masthead
 * skip and pass/fail rule, so gold files of the reference's regression
 * tests can be checked against results written here.
 */
#ifndef DICEGPU_RESULTS_H
#define DICEGPU_RESULTS_H

#include <stddef.h>
#include <stdint.h>

#include "dicegpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dicegpu_output dicegpu_output;

/* What the information block reports besides the params. */
typedef struct dicegpu_output_info {
  const char* ref_image;     /* "*** Reference image: %s " */
  const char* def_image;     /* "*** Deformed image: %s " (the first frame's) */
  const char* version;       /* masthead version text (the reference's git sha1) */
  int32_t subset_size;       /* "*** Subset size: %i" (-1 when none was given) */
  int32_t step_size_x;       /* -1: not a regular grid */
  int32_t step_size_y;
  int32_t strain_window;     /* -1: N/A */
  int32_t incremental;       /* use_incremental_formulation (also on when the params set it) */
  int32_t sort_rows;         /* sort_txt_output: per-frame files' rows by x, then y */
  const char* initialization_method;  /* reported initializer name; NULL: USE_FIELD_VALUES */
} dicegpu_output_info;

/* An output specification: `fields` lists the columns by their reference
 * names separated by commas or blanks (COORDINATE_X, DISPLACEMENT_X,
 * ROTATION_Z, NORMAL_STRAIN_X, SHEAR_STRAIN_XY, QUAD_A..QUAD_L, SIGMA, GAMMA,
 * BETA, OMEGA, NOISE_LEVEL, CONTRAST_LEVEL, ACTIVE_PIXELS, MATCH,
 * ITERATIONS, STATUS_FLAG, CONDITION_NUMBER, FIELD_1..FIELD_10,
 * VSG_STRAIN_XX .. VSG_DVDY, ...), or is
 * NULL for the default specification (Output_Spec without an output_spec
 * list).  A known field this library does not compute prints 0, as the
 * reference prints fields it has not allocated; an unknown name is
 * DICEGPU_ERR_ARG.  delimiter NULL means " ". */
int dicegpu_output_create(const dicegpu_params* params, const char* fields, const char* delimiter,
                          int omit_row_id, const dicegpu_output_info* info, dicegpu_output** out);
int dicegpu_output_destroy(dicegpu_output* o);
/* The image names of the information block (per-frame files report each
 * frame's deformed image); NULL leaves a name unchanged. */
int dicegpu_output_set_images(dicegpu_output* o, const char* ref_image, const char* def_image);
int dicegpu_output_num_fields(const dicegpu_output* o, int* n);

/* Text of the information block, the header row (row id label, e.g.
 * "FRAME" or "SUBSET_ID") and one row (a DICEGPU_FIELD_STRIDE field row, an
 * optional DICEGPU_UNCERTAINTY_STRIDE row for FIELD_1..FIELD_7 and an
 * optional DICEGPU_VSG_STRIDE row for the VSG columns).  Writes
 * at most cap bytes including the terminating 0 and sets *len to the full
 * length (without the 0). */
int dicegpu_output_info_text(const dicegpu_output* o, char* buf, size_t cap, size_t* len);
int dicegpu_output_header_text(const dicegpu_output* o, const char* row_id, char* buf, size_t cap, size_t* len);
int dicegpu_output_row_text(const dicegpu_output* o, int row_index, const double* fields, const double* unc,
                            const double* vsg, char* buf, size_t cap, size_t* len);

/* Schema::write_output after a frame: n subsets' field rows (and optional
 * uncertainty and VSG rows).  separate_files = 1: one file per subset,
 * <folder><prefix>_<id>.txt with the id zero-padded to the digits of n,
 * created with the information block and header at frame == first_frame and
 * appended to after; 0: one file per frame, <folder><prefix>_<frame>.txt
 * zero-padded to the digits of first_frame + num_frames, rows by subset id
 * (or by x, then y, with info.sort_rows). */
int dicegpu_output_write_frame(const dicegpu_output* o, const char* folder, const char* prefix, int frame,
                               int first_frame, int num_frames, int n, const double* fields, const double* unc,
                               const double* vsg, int separate_files);

/* DICe_Diff: compares result file b against gold file a.  rel_tol (-t),
 * floor (-f; use_floor 0 when not given), numerical_only (-n),
 * num_procs (-p; b is then the base name of the parallel pieces).  Returns 0
 * on success with *failed = the number of differing lines (0: "TEST PASSED");
 * the report of differing lines goes to report (cap bytes) when given. */
int dicegpu_diff_files(const char* a, const char* b, double rel_tol, double floor, int use_floor,
                       int numerical_only, int num_procs, int* failed, char* report, size_t cap);
/* The same on texts in memory (serial comparison). */
int dicegpu_diff_text(const char* a, size_t a_len, const char* b, size_t b_len, double rel_tol, double floor,
                      int use_floor, int numerical_only, int* failed, char* report, size_t cap);

#ifdef __cplusplus
}
#endif

#endif /* DICEGPU_RESULTS_H */
