// dg_vsg.cuh -- virtual strain gauge (VSG) strain of the subset field.
//
// VSG_Strain_Post_Processor::execute (DICe_PostProcessor.cpp:931-1130): for
// every subset, the subsets whose centres lie within window/2 (the kd-tree
// radius search of Post_Processor::initialize_neighborhood, :207-231: float
// squared distance < r^2 + 1e-5) and have sigma >= 0 fit u and v by planes
// [1, dx, dy] in double; the slopes give du/dx .. dv/dy and the
// Green-Lagrange strains.  Fewer than three valid neighbours, an invalid
// subset, or a reciprocal condition number below 1e-12 give zeros and
// MATCH = -1.  Field values enter as the reference's floats; results are
// rounded to float as the reference stores them.
//
// The neighbours come from a uniform grid of cell size >= the radius (3 x 3
// cells cover the disc) whose per-subset floats are packed in cell order
// (vsg_pack_kernel).  A warp accumulates the twelve double sums of X^T X,
// X^T u and X^T v for 32 subsets in turn, then each lane solves one
// subset's 3 x 3 system by LU with partial pivoting and an explicit inverse
// (the reference's GETRF / GETRI).
// The condition number is computed exactly where the reference estimates it
// (GECON); the two differ only for nearly collinear neighbourhoods.
#pragma once
#include <cstdint>

#include "dicegpu.h"

struct VsgArgs {
  double* fields;            // n x DICEGPU_FIELD_STRIDE (MATCH set to -1 where the fit fails)
  int n;
  const int32_t* cell_off;   // [ncx * ncy + 1] into cell_pts / packed
  const int32_t* cell_pts;   // subset indices grouped by cell
  const int32_t* pos_of;     // position of each subset in cell order
  float4* packed;            // per position: x (NaN when sigma < 0), y, u, v as floats
  int ncx, ncy;
  float x0, y0, cell;        // grid origin and cell size
  float r2;                  // r^2 + 1e-5
  double* out;               // n x DICEGPU_VSG_STRIDE
};

// The per-subset values the fits read, as the reference's floats, packed in
// cell order so that a cell's candidates are one coalesced run of 16-byte
// loads.  An invalid subset (sigma < 0) gets x = NaN, which fails the
// distance test exactly as the reference's validity test excludes it.
__global__ void __launch_bounds__(256) vsg_pack_kernel(VsgArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const double* f = a.fields + (size_t)i * DICEGPU_FIELD_STRIDE;
    const bool valid = (float)f[DICEGPU_F_SIGMA] >= 0.0f;
    a.packed[a.pos_of[i]] = make_float4(valid ? (float)f[DICEGPU_F_COORD_X] : __int_as_float(0x7fc00000),
                                        (float)f[DICEGPU_F_COORD_Y], (float)f[DICEGPU_F_DISP_X],
                                        (float)f[DICEGPU_F_DISP_Y]);
  }
}

__device__ __forceinline__ double vsg_warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// LU with partial pivoting and the inverse of a 3 x 3; false on a zero pivot
__device__ inline bool vsg_inverse3(const double A_in[3][3], double inv[3][3]) {
  double A[3][3];
  int piv[3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = A_in[i][j];
  for (int k = 0; k < 3; ++k) {
    int p = k;
    for (int i = k + 1; i < 3; ++i)
      if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
    piv[k] = p;
    if (A[p][k] == 0.0) return false;
    if (p != k)
      for (int j = 0; j < 3; ++j) { const double t = A[k][j]; A[k][j] = A[p][j]; A[p][j] = t; }
    for (int i = k + 1; i < 3; ++i) {
      A[i][k] = __ddiv_rn(A[i][k], A[k][k]);
      for (int j = k + 1; j < 3; ++j) A[i][j] = __dsub_rn(A[i][j], __dmul_rn(A[i][k], A[k][j]));
    }
  }
  for (int c = 0; c < 3; ++c) {
    double b[3] = {0.0, 0.0, 0.0};
    b[c] = 1.0;
    for (int k = 0; k < 3; ++k) { const double t = b[k]; b[k] = b[piv[k]]; b[piv[k]] = t; }
    for (int i = 1; i < 3; ++i)
      for (int j = 0; j < i; ++j) b[i] = __dsub_rn(b[i], __dmul_rn(A[i][j], b[j]));
    for (int i = 2; i >= 0; --i) {
      for (int j = i + 1; j < 3; ++j) b[i] = __dsub_rn(b[i], __dmul_rn(A[i][j], b[j]));
      b[i] = __ddiv_rn(b[i], A[i][i]);
    }
    for (int i = 0; i < 3; ++i) inv[i][c] = b[i];
  }
  return true;
}

__device__ inline double vsg_norm1(const double M[3][3]) {
  double a = 0.0;
  for (int j = 0; j < 3; ++j) a = fmax(a, fabs(M[0][j]) + fabs(M[1][j]) + fabs(M[2][j]));
  return a;
}

// One warp per batch of 32 subsets.  For each subset of the batch the lanes
// take its candidates in turn (the three cells of a grid row are one
// contiguous run of the packed array) and the twelve double sums are reduced
// across the warp; lane k keeps subset k's sums, and the 32 solves then run
// in parallel, one per lane.
__global__ void __launch_bounds__(256) vsg_kernel(VsgArgs a) {
  const int lane = threadIdx.x & 31;
  const int nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < a.n; base += nwarps * 32) {
    const int cnt = min(32, a.n - base);
    double m[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) m[k] = 0.0;
    int mvalid = 0;
    bool mself = false;
    for (int k = 0; k < cnt; ++k) {
      const int i = base + k;
      const double* fi = a.fields + (size_t)i * DICEGPU_FIELD_STRIDE;
      const float xi = (float)fi[DICEGPU_F_COORD_X], yi = (float)fi[DICEGPU_F_COORD_Y];
      const int gx = (int)floorf((xi - a.x0) / a.cell), gy = (int)floorf((yi - a.y0) / a.cell);
      // sums: n, dx, dy, dx dx, dx dy, dy dy, u, dx u, dy u, v, dx v, dy v
      double s[12];
#pragma unroll
      for (int q = 0; q < 12; ++q) s[q] = 0.0;
      int valid = 0;
      const int cx0 = max(gx - 1, 0), cx1 = min(gx + 1, a.ncx - 1);
      for (int cy = max(gy - 1, 0); cy <= min(gy + 1, a.ncy - 1); ++cy) {
        const int t1 = a.cell_off[cy * a.ncx + cx1 + 1];
        for (int t = a.cell_off[cy * a.ncx + cx0] + lane; t < t1; t += 32) {
          const float4 pj = __ldg(a.packed + t);
          const float ex = __fsub_rn(xi, pj.x), ey = __fsub_rn(yi, pj.y);
          const float d2 = __fadd_rn(__fmul_rn(ex, ex), __fmul_rn(ey, ey));
          if (!(d2 < a.r2)) continue;   // also an invalid neighbour (x = NaN)
          const double dx = (double)__fsub_rn(pj.x, xi), dy = (double)__fsub_rn(pj.y, yi);
          const double u = (double)pj.z, v = (double)pj.w;
          ++valid;
          s[0] += 1.0; s[1] += dx; s[2] += dy;
          s[3] = fma(dx, dx, s[3]); s[4] = fma(dx, dy, s[4]); s[5] = fma(dy, dy, s[5]);
          s[6] += u; s[7] = fma(dx, u, s[7]); s[8] = fma(dy, u, s[8]);
          s[9] += v; s[10] = fma(dx, v, s[10]); s[11] = fma(dy, v, s[11]);
        }
      }
#pragma unroll
      for (int q = 0; q < 12; ++q) s[q] = vsg_warp_sum(s[q]);
      for (int o = 16; o > 0; o >>= 1) valid += __shfl_xor_sync(0xffffffffu, valid, o);
      if (lane == k) {
#pragma unroll
        for (int q = 0; q < 12; ++q) m[q] = s[q];
        mvalid = valid;
        mself = (float)fi[DICEGPU_F_SIGMA] >= 0.0f;
      }
    }
    if (lane >= cnt) continue;
    const int i = base + lane;
    double* o = a.out + (size_t)i * DICEGPU_VSG_STRIDE;
    double r[7] = {0, 0, 0, 0, 0, 0, 0};
    bool ok = mself && mvalid >= 3;
    if (ok) {
      const double XtX[3][3] = {{m[0], m[1], m[2]}, {m[1], m[3], m[4]}, {m[2], m[4], m[5]}};
      double inv[3][3];
      ok = vsg_inverse3(XtX, inv);
      if (ok) ok = !(1.0 / (vsg_norm1(XtX) * vsg_norm1(inv)) < 1.0e-12);
      if (ok) {
        const double Xu[3] = {m[6], m[7], m[8]}, Xv[3] = {m[9], m[10], m[11]};
        double cu[3], cv[3];
        for (int p = 0; p < 3; ++p) {
          cu[p] = inv[p][0] * Xu[0] + inv[p][1] * Xu[1] + inv[p][2] * Xu[2];
          cv[p] = inv[p][0] * Xv[0] + inv[p][1] * Xv[1] + inv[p][2] * Xv[2];
        }
        const double dudx = cu[1], dudy = cu[2], dvdx = cv[1], dvdy = cv[2];
        r[0] = (float)(0.5 * (2.0 * dudx + dudx * dudx + dvdx * dvdx));
        r[1] = (float)(0.5 * (2.0 * dvdy + dudy * dudy + dvdy * dvdy));
        r[2] = (float)(0.5 * (dudy + dvdx + dudx * dudy + dvdx * dvdy));
        r[3] = (float)dudx; r[4] = (float)dudy; r[5] = (float)dvdx; r[6] = (float)dvdy;
      }
    }
    for (int k = 0; k < 7; ++k) o[k] = r[k];
    o[DICEGPU_VSG_NEIGHBORS] = mvalid;
    if (!ok) a.fields[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_MATCH] = -1.0;
  }
}

// k nearest neighbourhoods (a negative window: Post_Processor::
// initialize_neighborhood's knnSearch, DICe_PostProcessor.cpp:185-205): the
// k nearest subsets, valid or not, listed per subset in ascending float
// squared distance (ties by index) by the host.  One thread per subset
// forms the same sums as the oracle, neighbour by neighbour in list order,
// each product and sum rounded on its own; the nearest (the subset itself)
// must be valid, as the reference tests neighbour 0.
struct VsgKnnArgs {
  double* fields;
  int n, k;
  const int32_t* nbr;        // n x k neighbour indices
  double* out;               // n x DICEGPU_VSG_STRIDE
};

__global__ void __launch_bounds__(256) vsg_knn_kernel(VsgKnnArgs a) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const int32_t* nb = a.nbr + (size_t)i * a.k;
    const double* fi = a.fields + (size_t)i * DICEGPU_FIELD_STRIDE;
    const float xi = (float)fi[DICEGPU_F_COORD_X], yi = (float)fi[DICEGPU_F_COORD_Y];
    int valid = 0;
    for (int q = 0; q < a.k; ++q) valid += (float)a.fields[(size_t)nb[q] * DICEGPU_FIELD_STRIDE + DICEGPU_F_SIGMA] >= 0.0f;
    bool ok = valid >= 3 && (float)a.fields[(size_t)nb[0] * DICEGPU_FIELD_STRIDE + DICEGPU_F_SIGMA] >= 0.0f;
    double r[7] = {0, 0, 0, 0, 0, 0, 0};
    if (ok) {
      double XtX[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Xu[3] = {0, 0, 0}, Xv[3] = {0, 0, 0};
      for (int q = 0; q < a.k; ++q) {
        const double* fj = a.fields + (size_t)nb[q] * DICEGPU_FIELD_STRIDE;
        if (!((float)fj[DICEGPU_F_SIGMA] >= 0.0f)) continue;
        const double row[3] = {1.0, (double)__fsub_rn((float)fj[DICEGPU_F_COORD_X], xi),
                               (double)__fsub_rn((float)fj[DICEGPU_F_COORD_Y], yi)};
        const double u = (double)(float)fj[DICEGPU_F_DISP_X], v = (double)(float)fj[DICEGPU_F_DISP_Y];
#pragma unroll
        for (int p = 0; p < 3; ++p) {
#pragma unroll
          for (int b = 0; b < 3; ++b) XtX[p][b] = __dadd_rn(XtX[p][b], __dmul_rn(row[p], row[b]));
          Xu[p] = __dadd_rn(Xu[p], __dmul_rn(row[p], u));
          Xv[p] = __dadd_rn(Xv[p], __dmul_rn(row[p], v));
        }
      }
      double inv[3][3];
      ok = vsg_inverse3(XtX, inv);
      if (ok) ok = !(1.0 / (vsg_norm1(XtX) * vsg_norm1(inv)) < 1.0e-12);
      if (ok) {
        double cu[3], cv[3];
        for (int p = 0; p < 3; ++p) {
          cu[p] = inv[p][0] * Xu[0] + inv[p][1] * Xu[1] + inv[p][2] * Xu[2];
          cv[p] = inv[p][0] * Xv[0] + inv[p][1] * Xv[1] + inv[p][2] * Xv[2];
        }
        const double dudx = cu[1], dudy = cu[2], dvdx = cv[1], dvdy = cv[2];
        r[0] = (float)(0.5 * (2.0 * dudx + dudx * dudx + dvdx * dvdx));
        r[1] = (float)(0.5 * (2.0 * dvdy + dudy * dudy + dvdy * dvdy));
        r[2] = (float)(0.5 * (dudy + dvdx + dudx * dudy + dvdx * dvdy));
        r[3] = (float)dudx; r[4] = (float)dudy; r[5] = (float)dvdx; r[6] = (float)dvdy;
      }
    }
    double* o = a.out + (size_t)i * DICEGPU_VSG_STRIDE;
    for (int q = 0; q < 7; ++q) o[q] = r[q];
    o[DICEGPU_VSG_NEIGHBORS] = valid;
    if (!ok) a.fields[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_MATCH] = -1.0;
  }
}
