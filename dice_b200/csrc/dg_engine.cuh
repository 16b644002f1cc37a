// dg_engine.cuh -- the per-subset correlation engine, one warp per subset.
//
// Mirrors Schema::generic_correlation_routine (DICe_Schema.cpp:2026-2368)
// with the field-value initializer (the subset's own row, or its
// neighbour's):
//   initial guess -> Gauss-Newton (Objective_ZNSSD::computeUpdateFast,
//   DICe_Objective.cpp:430-657) and/or Nelder-Mead (Simplex::minimize,
//   DICe_Simplex.cpp:60-277) -> jump test -> sigma -> gamma -> record_step.
//
// Data flow per Gauss-Newton iteration (one "pass" over the subset pixels):
//   lane <- pixel;  warp (map) -> round + border test -> interpolation of
//   I (+ Gx, Gy) -> residual vector r (FP32) -> v = [r, G-F, 1]
//   -> sum v v^T with FP64 tensor-core mma (exact products of FP32 values,
//   FP64 sums).  The 8x8 (affine) / 16x16 (quadratic) result holds
//   H = sum r r^T, sum r (G-F), sum r, sum (G-F) and the active count, from
//   which the reference's q = sum r ((G - meanG) - (F - meanF)) follows as
//   sum r (G-F) - (meanG - meanF) sum r.
#pragma once

#include "dg_pass.cuh"

namespace dg {

// MODE_CORRELATE: Schema::execute_correlation for each subset.  The other
// modes run one Objective entry point on the parameters of each field row:
// gamma, Gauss-Newton alone, the simplex alone, sigma.
enum { MODE_CORRELATE = 0, MODE_GAMMA = 1, MODE_GN = 2, MODE_SIMPLEX = 3, MODE_SIGMA = 4 };

struct FrameArgs {
  DevParams P;
  DevImage ref;
  DevImage def;
  DevGeometry geo;
  double* fields;        // n x DICEGPU_FIELD_STRIDE
  int n;
  int first_frame;
  int mode;
  int plain_index;       // >= 0: this launch processes only that subset (plain path)
  double* gamma_out;     // MODE_GAMMA output
  int* work_counter;     // queue heads: one (queue_mode 0) or one per CTA (1)
  int queue_mode;
  int chunk;             // consecutive subsets per queue chunk (queue_mode 1)
  int* status;           // device error word
  int32_t* passes_out;   // optional: pixel passes executed per subset (GN + simplex + epilogue)
  double* unc;           // optional: n x DICEGPU_UNCERTAINTY_STRIDE uncertainty fields
  int32_t* iter_out;     // MODE_GN / MODE_SIMPLEX: iterations per subset
  int32_t* status_out;   // MODE_GN / MODE_SIMPLEX: Status_Flag per subset
  double* noise_out;     // MODE_SIGMA: noise_std_dev per subset (sigma goes to gamma_out)
  const int32_t* order;  // optional: the subsets of this launch (a tracking wave), n_order of them
  int n_order;
  int evolve;            // turn on visible inactive pixels of evolving subsets after success
  const int32_t* neigh;  // neighbour initialization this frame: NEIGHBOR_ID per subset
  const double* nsnap;   // the fields at frame start (neighbours with a higher index)
};

// Image_::interpolate_keys_fourth (DICe_Image.cpp:890-924), intensity only:
// the bilinear value (Image_::interpolate_bilinear, :432-445) near the
// border, the 6 x 6 Keys sum (rows outer) elsewhere.
__device__ __forceinline__ float keys_intensity(const DevImage& im, float lx, float ly) {
  const int w = im.w, h = im.h;
  const float* __restrict__ I = im.I;
  // both range tests are written so that a NaN coordinate returns 0
  if (!(lx > 2.5f && lx < (float)w - 3.5f && ly > 2.5f && ly < (float)h - 3.5f)) {
    if (!(lx >= 0.0f && lx < (float)w - 1.5f && ly >= 0.0f && ly < (float)h - 1.5f)) return 0.0f;
    const int x1 = (int)lx, x2 = x1 + 1, y1 = (int)ly, y2 = y1 + 1;
    return __ldg(I + (size_t)y1 * w + x1) * ((float)x2 - lx) * ((float)y2 - ly) +
           __ldg(I + (size_t)y1 * w + x2) * (lx - (float)x1) * ((float)y2 - ly) +
           __ldg(I + (size_t)y2 * w + x2) * (lx - (float)x1) * (ly - (float)y1) +
           __ldg(I + (size_t)y2 * w + x1) * ((float)x2 - lx) * (ly - (float)y1);
  }
  const int ix = (int)lx, iy = (int)ly;
  float wx[6], wy[6];
  keys_weights(lx - (float)ix, wx);
  keys_weights(ly - (float)iy, wy);
  float v = 0.0f;
#pragma unroll
  for (int m = 0; m < 6; ++m) {
    const float* row = I + (size_t)(iy - 2 + m) * w + ix - 2;
#pragma unroll
    for (int n = 0; n < 6; ++n) v += wy[m] * wx[n] * __ldg(row + n);
  }
  return v;
}

struct AffineStep {
  float upd[6];   // parameter update per slot (0 for disabled slots)
  float cond;     // 2x2 condition number of the displacement block
};

// Gauss-Newton step of the affine system, computed by every lane on its own
// copy (no shuffles, all in registers).  `M` is the accumulated 8x8 matrix of
// [r(6 slots), G-F, 1]; `em` the mask of enabled slots.  Mirrors
// DICe_Objective.cpp:548-607: LM penalty, the 2x2 condition number in the
// reference's float/double mix, LU with partial pivoting in DGETRF order
// (first maximal pivot, reciprocal scaling, rank-1 updates), then
// update = -H^-1 q, or -LU q when a pivot is exactly zero (DGETRI returns
// early and the factors are used as the inverse).
static __device__ __noinline__ AffineStep solve_affine(const double* __restrict__ M, double cshift,
                                                unsigned em, float lm_alpha) {
  double H[6][6], q[6], q0[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    const bool ei = (em >> i) & 1u;
#pragma unroll
    for (int j = 0; j < 6; ++j) {
      const bool ej = (em >> j) & 1u;
      H[i][j] = (ei && ej) ? M[i * 8 + j] : (i == j ? 1.0 : 0.0);
    }
    q[i] = ei ? M[i * 8 + 6] - cshift * M[i * 8 + 7] : 0.0;
    q0[i] = q[i];
  }
  if (lm_alpha > 0.0f) {
    H[0][0] += (double)lm_alpha;
    H[1][1] += (double)lm_alpha;
  }
  AffineStep out;
  {
    const double nsq = H[0][0] * H[0][0] + H[0][1] * H[0][1] + H[1][0] * H[1][0] + H[1][1] * H[1][1];
    const float det_h = (float)(H[0][0] * H[1][1] - H[1][0] * H[0][1]);
    const float norm_H = (float)sqrt(nsq);
    float cond = -1.0f;
    if (det_h != 0.0f) {
      const float dd = __fmul_rn(det_h, det_h);
      cond = norm_H * (float)sqrt((1.0 / (double)dd) * nsq);
    }
    out.cond = cond;
  }
  int info = 0;
#pragma unroll
  for (int j = 0; j < 6; ++j) {
    int p = j;
    double best = fabs(H[j][j]);
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
      const double a = fabs(H[i][j]);
      if (a > best) { best = a; p = i; }
    }
    double pv = H[j][j];
#pragma unroll
    for (int i = j + 1; i < 6; ++i)
      if (i == p) pv = H[i][j];
    if (pv != 0.0) {
#pragma unroll
      for (int i = j + 1; i < 6; ++i) {
        if (i == p) {
#pragma unroll
          for (int k = 0; k < 6; ++k) {
            const double t = H[j][k];
            H[j][k] = H[i][k];
            H[i][k] = t;
          }
          const double t = q[j];
          q[j] = q[i];
          q[i] = t;
        }
      }
      const double r = 1.0 / pv;
#pragma unroll
      for (int i = j + 1; i < 6; ++i) H[i][j] *= r;
    } else if (info == 0) {
      info = j + 1;
    }
#pragma unroll
    for (int i = j + 1; i < 6; ++i) {
#pragma unroll
      for (int k = j + 1; k < 6; ++k) H[i][k] -= H[i][j] * H[j][k];
      q[i] -= H[i][j] * q[j];
    }
  }
  if (info == 0) {
    double x[6];
#pragma unroll
    for (int j = 5; j >= 0; --j) {
      double s = q[j];
#pragma unroll
      for (int k = j + 1; k < 6; ++k) s -= H[j][k] * x[k];
      x[j] = s / H[j][j];
    }
#pragma unroll
    for (int i = 0; i < 6; ++i) out.upd[i] = (float)(-x[i]);
  } else {
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      float u = 0.0f;
#pragma unroll
      for (int j = 0; j < 6; ++j) u = (float)((double)u + H[i][j] * (-1.0) * q0[j]);
      out.upd[i] = u;
    }
  }
  return out;
}

struct SubsetRef {
  int idx, cx, cy, npix;
  int off;          // list offset (-1 for squares)
  float K;          // intensity shift for the moment sums
  bool masked;      // has an obstruction bitmap, blocked polygons or evolution state
  bool evo;         // evolving: its list keeps inactive pixels (per-pixel state)
  int nact;         // pixels with is_active set (npix unless evolving)
};

template <int SHAPE, int INTERP, bool DEFGRAD, bool MASK>
struct Engine {
  using L = Layout<SHAPE>;
  const FrameArgs& A;
  const int lane;
  int npass_ = 0;   // pixel passes of the current subset (for work accounting)

  __device__ explicit Engine(const FrameArgs& a) : A(a), lane(threadIdx.x & 31) {}

  __device__ __forceinline__ void pixel_xy(const SubsetRef& sb, int p, int& x, int& y) const {
    if (sb.off < 0) {
      const int side = 2 * A.geo.half + 1;
      const int row = p / side, col = p - row * side;
      x = sb.cx - A.geo.half + col;
      y = sb.cy - A.geo.half + row;
    } else {
      x = __ldg(A.geo.px + sb.off + p);
      y = __ldg(A.geo.py + sb.off + p);
    }
    x = x < 0 ? 0 : x;   // Subset ctors clamp negative coordinates (DICe_Subset.cpp:66-68, :100-101)
    y = y < 0 ? 0 : y;
  }

  // One pass over the subset at the parameters in `slots` (see subset_pass).
  template <bool ACC_H, bool GRADS, bool MOMENTS>
  __device__ __forceinline__ PassOut pass(const SubsetRef& sb, const float* slots, double* /*C*/) {
    PassInMasked in;
    in.def = A.def;
    in.refI = A.ref.I;
    in.refgx = A.ref.gx;
    in.refgy = A.ref.gy;
    in.refw = A.ref.w;
    in.reflim = (long)A.ref.w * A.ref.h;
    in.px = A.geo.px;
    in.py = A.geo.py;
    in.half = A.geo.half;
    in.cx = sb.cx;
    in.cy = sb.cy;
    in.npix = sb.npix;
    in.off = sb.off;
    in.K = sb.K;
    MapConst k;
    make_mapconst<SHAPE>(slots, !DEFGRAD, (float)sb.cx, (float)sb.cy, k);
    if (MASK && sb.masked) {
      in.mdesc = A.geo.mask_desc + (size_t)sb.idx * DG_MASK_DESC;
      in.mbits = A.geo.mask_bits;
      in.bpoly = A.geo.blocked_poly;
      in.bvx = A.geo.blocked_vx;
      in.bvy = A.geo.blocked_vy;
      in.pflag = sb.evo ? A.geo.pix_flag : nullptr;
      in.pfv = sb.evo ? A.geo.pix_f : nullptr;
      return subset_pass<SHAPE, INTERP, DEFGRAD, ACC_H, GRADS, MOMENTS, true>(in, k);
    }
    return subset_pass<SHAPE, INTERP, DEFGRAD, ACC_H, GRADS, MOMENTS, false>(static_cast<const PassIn&>(in), k);
  }

  // Objective::gamma from the moments (Subset::gamma, DICe_Subset.cpp:323-340):
  // gamma = sum ((G-mG)/|G-mG| - (F-mF)/|F-mF|)^2 = 2 - 2 cov / (|G-mG| |F-mF|).
  __device__ float gamma_from(const PassOut& o, int npix) const {
    if (o.n == 0) return -1.0f;
    const double n = (double)o.n;
    const double sgg = o.sG2 - o.sG * o.sG / n;
    const double sff = o.sF2 - o.sumF * o.sumF / n;
    const double sgf = o.sGF - o.sG * o.sumF / n;
    if (!(sgg > 0.0) || !(sff > 0.0)) return -1.0f;
    double g = 2.0 - 2.0 * sgf / sqrt(sgg * sff);
    if (g < 0.0) g = 0.0;
    float gf = (float)g;
    if (A.P.normalize_gamma && npix > 0) gf /= (float)npix;
    return gf;
  }

  __device__ float eval_gamma(const SubsetRef& sb, const float* slots, PassOut* out = nullptr) {
    PassOut o = pass<false, false, true>(sb, slots, nullptr);
    if (out) *out = o;
    ++npass_;
    return gamma_from(o, sb.nact);
  }

  __device__ void compact_to_slots(const float* comp, float* slots, const float* base) const {
#pragma unroll
    for (int i = 0; i < 12; ++i) slots[i] = base[i];
    for (int k = 0; k < A.P.N; ++k) slots[A.P.slot[k]] = comp[k];
  }

  __device__ __forceinline__ unsigned enabled_mask() const {
    unsigned em = 0;
    for (int k = 0; k < A.P.N; ++k) em |= 1u << A.P.slot[k];
    return em;
  }

  // Objective::computeUncertaintyFields (DICe_Objective.cpp:193-299) after a
  // converged Gauss-Newton step, without an image deformer (exact motion 0).
  // `before` holds the parameters of the last pass, whose gradients the
  // reference's subset still holds; `after` the converged parameters (u, v).
  // Every subset pixel takes part.  A pixel outside the 4-pixel border at the
  // last pass takes the reference-image gradient (the reference keeps the
  // gradient of the last pass in which that pixel was inside, which differs
  // only for subsets reaching the border).  Sums in FP64; the fields are
  // rounded to float like the reference's float fields.
  // Arguments travel by value (registers): a pointer to the caller's arrays
  // would move them to local memory for the whole Gauss-Newton loop.
  struct Slots {
    float s[12];
  };
  __device__ __noinline__ void write_uncertainty(const SubsetRef sb, const Slots before,
                                                 const Slots after) {
    const double* f = A.fields + (size_t)sb.idx * DICEGPU_FIELD_STRIDE;
    const float ucx = (float)f[DICEGPU_F_COORD_X], ucy = (float)f[DICEGPU_F_COORD_Y];
    MapConst kb, ka;
    const float fcx = (float)sb.cx, fcy = (float)sb.cy;
    make_mapconst<SHAPE>(before.s, false, fcx, fcy, kb);
    make_mapconst<SHAPE>(after.s, false, ucx, ucy, ka);
    float u, v, t;
    map_to_u_v_theta<SHAPE>(ka, ucx, ucy, u, v, t);
    const int W = A.def.w, H = A.def.h;
    const long rlim = (long)A.ref.w * A.ref.h;
    double s_g2 = 0.0, s_uhat = 0.0, s_ug = 0.0, s_jg = 0.0, s_r = 0.0;
    for (int p = lane; p < sb.npix; p += 32) {
      int x, y;
      pixel_xy(sb, p, x, y);
      const long ri = (long)y * A.ref.w + x;
      const bool rin = ri < rlim;
      float gx = rin ? __ldg(A.ref.gx + ri) : 0.0f;
      float gy = rin ? __ldg(A.ref.gy + ri) : 0.0f;
      if (DEFGRAD) {
        float mx, my, Dx, Dy;
        map_offset<SHAPE>(kb, __fsub_rn((float)x, fcx), __fsub_rn((float)y, fcy), fcx, fcy, mx, my,
                          Dx, Dy);
        const int px = round_pixel(mx), py = round_pixel(my);
        if (!(px < 4 || px >= W - 4 || py < 4 || py >= H - 4)) {
          float G;
          interp_interior<INTERP, true>(A.def, mx, my, G, gx, gy);
        }
      }
      const float g2 = gx * gx + gy * gy;
      s_g2 += (double)g2;
      s_uhat += (double)(u * u + v * v);
      const float inv_g2 = g2 < 1.0e-4f ? 0.0f : (float)(1.0 / (double)g2);
      const float a = u * gx + v * gy;
      s_ug += (double)(a * a * inv_g2);
      const float j = v * gx - u * gy;
      s_jg += (double)(j * j * inv_g2);
      const float r0 = rin ? __ldg(A.ref.I + ri) : 0.0f;
      const float sub_r = keys_intensity(A.def, (float)x + u, (float)y + v) - r0;
      const float sub_e = keys_intensity(A.def, (float)x, (float)y) - r0;
      const float d = sub_r - sub_e;
      s_r += (double)(d * d * inv_g2);
    }
    s_g2 = warp_sum(s_g2);
    s_uhat = warp_sum(s_uhat);
    s_ug = warp_sum(s_ug);
    s_jg = warp_sum(s_jg);
    s_r = warp_sum(s_r);
    if (lane == 0) {
      const float cos_hat = s_uhat == 0.0 ? 1.0f : (float)sqrt(s_ug / s_uhat);
      double* o = A.unc + (size_t)sb.idx * DICEGPU_UNCERTAINTY_STRIDE;
      o[DICEGPU_U_COS_THETA_HAT] = cos_hat;
      o[DICEGPU_U_COS_THETA] = 1.0;
      o[DICEGPU_U_ERROR_L2] = (float)sqrt(s_ug + s_jg);
      o[DICEGPU_U_RESIDUAL_ERROR] =
          cos_hat == 0.0f ? 0.0 : (double)(float)(1.0 / (double)cos_hat * (double)(float)sqrt(s_r));
      o[DICEGPU_U_ERROR_GRAD_PHI] = (float)sqrt(s_ug);
      o[DICEGPU_U_RESIDUAL] = (float)sqrt(s_r);
      o[DICEGPU_U_SSSIG] = (float)((1.0 + s_g2) / (sb.npix ? (double)sb.npix : 1.0));
    }
  }

  // Subset::turn_on_previously_obstructed_pixels (DICe_Subset.cpp:506-520)
  // after a successful solve (DICe_Schema.cpp:2354-2360): each inactive
  // pixel that the last deformed-state initialisation (the final parameters,
  // Objective::gamma) left visible takes the deformed intensity interpolated
  // there as its reference intensity and becomes active.
  __device__ __noinline__ void evolve(const SubsetRef sb, const Slots fin) {
    MapConst k;
    const float fcx = (float)sb.cx, fcy = (float)sb.cy;
    make_mapconst<SHAPE>(fin.s, !DEFGRAD, fcx, fcy, k);
    const int W = A.def.w, H = A.def.h;
    const MaskView mv(A.geo.mask_desc + (size_t)sb.idx * DG_MASK_DESC, A.geo.mask_bits, A.geo.blocked_poly,
                      A.geo.blocked_vx, A.geo.blocked_vy);
    int on = 0;
    for (int p = lane; p < sb.npix; p += 32) {
      uint8_t* st = A.geo.pix_flag + sb.off + p;
      if (*st != 0) continue;
      int x, y;
      pixel_xy(sb, p, x, y);
      float mx, my, Dx, Dy;
      map_offset<SHAPE>(k, __fsub_rn((float)x, fcx), __fsub_rn((float)y, fcy), fcx, fcy, mx, my, Dx, Dy);
      const int px = round_pixel(mx), py = round_pixel(my);
      if (px < 4 || px >= W - 4 || py < 4 || py >= H - 4 || mv.hides(px, py)) continue;
      float G, gx, gy;
      interp_interior<INTERP, false>(A.def, mx, my, G, gx, gy);
      A.geo.pix_f[sb.off + p] = G;
      *st = 2;
      ++on;
    }
    on = warp_sum_i(on);
    if (lane == 0 && on) A.geo.evo_nact[sb.idx] += on;
  }

  __device__ __forceinline__ void uncertainty_hook(const SubsetRef& sb, const float* before,
                                                   const float* after) {
    Slots b, a;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      b.s[i] = before[i];
      a.s[i] = after[i];
    }
    write_uncertainty(sb, b, a);
  }

  // --------------------------------------------------------------------------
  // Gauss-Newton (Objective_ZNSSD::computeUpdateFast).  `slots` in/out.
  // `meanF` is the reference mean at entry (Subset::mean(REF_INTENSITIES)).
  // --------------------------------------------------------------------------
  // meanF < 0 is never a valid "not given" marker for intensities, so the
  // all-pixel mean of a fresh subset is requested with `meanF_from_pass`.
  __device__ int gauss_newton(const SubsetRef& sb, float* slots, float meanF, bool meanF_from_pass,
                              int& num_iterations,
                              float& cond_out, PassOut& last) {
    const DevParams& P = A.P;
    const int N = P.N;
    float upd_old[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) upd_old[i] = 0.0f;
    double* M = warp_smem<SHAPE>()->M;
    int solve_it = 0;
    for (; solve_it <= P.max_fast; ++solve_it) {
      num_iterations = solve_it;
      DG_PT(t_pass);
      last = pass<true, true, false>(sb, slots, M);
      DG_PACC(1, t_pass);
      ++npass_;
      const int n = last.n;
      // Subset::mean(DEF_INTENSITIES): sum G / n over the active pixels
      const double sumG = M[L::ID * L::VW + L::IONE] + last.sumF + (double)n * (double)sb.K;
      const float meanG = n ? (float)(sumG / (double)n) : 0.0f;
      if (meanF_from_pass && solve_it == 0) {
        // Subset::mean(REF_INTENSITIES) at entry: every active pixel of a fresh subset
        meanF = sb.nact ? (float)((last.sumFall + (double)sb.nact * (double)sb.K) / (double)sb.nact)
                        : 0.0f;
      }
      const double cshift = (double)meanG - (double)meanF;
      if constexpr (SHAPE == DICEGPU_AFFINE_SF) {
        // Every lane solves the whole (padded) 6x6 system in registers: the
        // slots of disabled parameters get identity rows / columns and q = 0,
        // which leaves the LU of the enabled block (same pivots, same
        // operations) unchanged and gives them a zero update.
        const AffineStep stp = solve_affine(M, cshift, enabled_mask(), P.lm_alpha);
        const float* upd_s = stp.upd;
        cond_out = stp.cond;
        if (stp.cond > 1.0e12f) return DICEGPU_HESSIAN_SINGULAR;
        float old[12];
#pragma unroll
        for (int i = 0; i < 12; ++i) old[i] = slots[i];
#pragma unroll
        for (int s = 0; s < 6; ++s) {
          float u = upd_s[s];
          if (P.momentum != 0.0f) {
            u += P.momentum * upd_old[s];
            upd_old[s] = u;
          }
          slots[s] += u;   // disabled slots: u == 0
        }
        const float tol = P.fast_tol;
        bool conv = true;
        if (fabsf(slots[0] - old[0]) >= tol) conv = false;
        if (fabsf(slots[1] - old[1]) >= tol) conv = false;
        if (P.has_rot && fabsf(slots[2] - old[2]) >= tol) conv = false;
        if (conv) {
          if (A.unc && (A.mode == MODE_CORRELATE || A.mode == MODE_GN)) uncertainty_hook(sb, old, slots);
          break;
        }
        continue;
      }
      // lane i owns row i of [H | q] in the reference's compact order
      double h[L::NMAX];
      double qv = 0.0;
      const int si = lane < N ? P.slot[lane] : 0;
#pragma unroll
      for (int j = 0; j < L::NMAX; ++j) {
        h[j] = 0.0;
        if (j < N && lane < N) h[j] = M[si * L::VW + P.slot[j]];
      }
      if (lane < N) qv = M[si * L::VW + L::ID] - cshift * M[si * L::VW + L::IONE];
      // Levenberg-Marquardt penalty on the displacement diagonal (:548-553)
      if (P.lm_alpha > 0.0f) {
        if (lane == 0) h[0] += (double)P.lm_alpha;
        if (lane == 1) h[1] += (double)P.lm_alpha;
      }
      // 2x2 condition number of the displacement block (:558-564), in the
      // reference's mix of float and double
      const double H00 = __shfl_sync(FULL, h[0], 0), H01 = __shfl_sync(FULL, h[1], 0);
      const double H10 = __shfl_sync(FULL, h[0], 1), H11 = __shfl_sync(FULL, h[1], 1);
      const float det_h = (float)(H00 * H11 - H10 * H01);
      const double nsq = H00 * H00 + H01 * H01 + H10 * H10 + H11 * H11;
      const float norm_H = (float)sqrt(nsq);
      float cond = -1.0f;
      if (det_h != 0.0f) {
        const float dd = __fmul_rn(det_h, det_h);
        const float norm_Hi = (float)sqrt((1.0 / (double)dd) * nsq);
        cond = norm_H * norm_Hi;
      }
      cond_out = cond;
      // LU with partial pivoting (DGETRF order), q carried as an extra column
      const double q_orig = qv;
      int info = 0;
#pragma unroll
      for (int j = 0; j < L::NMAX; ++j) {
        if (j < N) {
          double a = (lane >= j && lane < N) ? fabs(h[j]) : -1.0;
          int pl = lane;
#pragma unroll
          for (int o = 16; o > 0; o >>= 1) {
            const double oa = __shfl_xor_sync(FULL, a, o);
            const int op = __shfl_xor_sync(FULL, pl, o);
            if (oa > a || (oa == a && op < pl)) { a = oa; pl = op; }
          }
          const double pv = __shfl_sync(FULL, h[j], pl);
          if (pv != 0.0) {
            if (pl != j) {
              const int src = lane == j ? pl : (lane == pl ? j : lane);
#pragma unroll
              for (int kx = 0; kx < L::NMAX; ++kx) h[kx] = __shfl_sync(FULL, h[kx], src);
              qv = __shfl_sync(FULL, qv, src);
            }
            const double rcp = 1.0 / pv;
            if (lane > j && lane < N) h[j] *= rcp;
          } else if (info == 0) {
            info = j + 1;
          }
#pragma unroll
          for (int kx = j + 1; kx < L::NMAX; ++kx) {
            const double prow = __shfl_sync(FULL, h[kx], j);
            if (kx < N && lane > j && lane < N) h[kx] -= h[j] * prow;
          }
          const double pq = __shfl_sync(FULL, qv, j);
          if (lane > j && lane < N) qv -= h[j] * pq;
        }
      }
      if (cond > 1.0e12f) return DICEGPU_HESSIAN_SINGULAR;
      float upd = 0.0f;
      if (info == 0) {
        // back substitution: x = U^-1 y, update = -x
        double x = 0.0;
#pragma unroll
        for (int j = L::NMAX - 1; j >= 0; --j) {
          if (j < N) {
            const double ujj = __shfl_sync(FULL, h[j], j);
            const double yj = __shfl_sync(FULL, qv, j);
            const double xj = yj / ujj;
            if (lane == j) x = xj;
            if (lane < j) qv -= h[j] * xj;
          }
        }
        upd = (float)(-x);
      } else {
        // DGETRI returns early on a zero pivot and the LU factors themselves
        // are applied to -q (:591, :605-607), accumulated in float
#pragma unroll
        for (int j = 0; j < L::NMAX; ++j) {
          const double qj = __shfl_sync(FULL, q_orig, j);
          if (j < N) upd = (float)((double)upd + h[j] * (-1.0) * qj);
        }
      }
      float old[12];
#pragma unroll
      for (int i = 0; i < 12; ++i) old[i] = slots[i];
#pragma unroll
      for (int kx = 0; kx < 12; ++kx) {
        float u = __shfl_sync(FULL, upd, kx);
        if (kx < N) {
          if (P.momentum != 0.0f) {
            u += P.momentum * upd_old[kx];
            upd_old[kx] = u;
          }
          slots[P.slot[kx]] += u;
        }
      }
      // test_for_convergence (affine: u, v, theta :433-459; quadratic: all)
      const float tol = P.fast_tol;
      bool conv = true;
      if (SHAPE == DICEGPU_QUADRATIC_SF) {
#pragma unroll
        for (int i = 0; i < 12; ++i)
          if (fabsf(slots[i] - old[i]) >= tol) conv = false;
      } else {
        if (fabsf(slots[0] - old[0]) >= tol) conv = false;
        if (fabsf(slots[1] - old[1]) >= tol) conv = false;
        if (P.has_rot && fabsf(slots[2] - old[2]) >= tol) conv = false;
      }
      if (conv) {
        if (A.unc && (A.mode == MODE_CORRELATE || A.mode == MODE_GN)) uncertainty_hook(sb, old, slots);
        break;
      }
    }
    if (solve_it > P.max_fast) return DICEGPU_MAX_ITERATIONS_REACHED;
    return DICEGPU_CORRELATION_SUCCESSFUL;
  }

  // --------------------------------------------------------------------------
  // Nelder-Mead (Simplex::minimize, DICe_Simplex.cpp:60-277).  Every lane runs
  // the same bookkeeping on its own private copy of the simplex (identical
  // values in all lanes, no shared state); the gamma evaluations are
  // warp-wide passes.  `slots` in/out: left at the last evaluated point, as
  // the reference's aliasing of variables and shape-function parameters
  // leaves it (DICe_LocalShapeFunction.h:259-261).  `lastp` receives that
  // point in slot form.
  // --------------------------------------------------------------------------
  __device__ int simplex(const SubsetRef& sb, float* slots, int& num_iterations, float* lastp) {
    const DevParams& P = A.P;
    const int nd = P.N;
    const int mpts = nd + 1;
    float base[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) base[i] = slots[i];
    float vars[12], init[12], pts[13][12], gv[13], psum[12], ptry[12];
    for (int kx = 0; kx < nd; ++kx) init[kx] = base[P.slot[kx]];
    auto evaluate = [&]() -> float {
      float cs[12];
      for (int kx = 0; kx < 12; ++kx) cs[kx] = kx < nd ? vars[kx] : 0.0f;
      compact_to_slots(cs, lastp, base);
      return eval_gamma(sb, lastp);
    };
    auto finish = [&]() {
      float cs[12];
      for (int kx = 0; kx < 12; ++kx) cs[kx] = kx < nd ? vars[kx] : 0.0f;
      compact_to_slots(cs, slots, base);
    };
    // initial simplex vertex_i = x0 + delta_i e_i (:82-107)
    for (int i = 0; i < mpts; ++i) {
      for (int j = 0; j < nd; ++j) {
        pts[i][j] = init[j];
        if (i > 0 && j == i - 1) pts[i][j] += P.deltas[i - 1];
        vars[j] = pts[i][j];
      }
      gv[i] = evaluate();
      if (i == 0 && gv[i] < P.skip_thr && gv[i] >= 0.0f) {
        num_iterations = 0;
        finish();
        return DICEGPU_CORRELATION_SUCCESSFUL;
      }
      for (int j = 0; j < nd; ++j) vars[j] = init[j];
    }
    for (int j = 0; j < nd; ++j) {
      float sum = 0.0f;
      for (int i = 0; i < mpts; ++i) sum += pts[i][j];
      psum[j] = sum;
    }
    int inhi = 0;
    float old_rtol = 0.0f, gamma_new = 0.0f, gamma_old = -1.0f;
    int gamma_repeats = 0;
    const float tiny = 1.0e-10f;
    int iteration = 0;
    for (iteration = 0; iteration < P.max_robust; iteration++) {
      if (iteration >= P.max_robust - 1) {
        num_iterations = iteration;
        finish();
        return DICEGPU_MAX_ITERATIONS_REACHED;
      }
      int ilo = 0;
      int ihi;
      if (gv[0] > gv[1]) { inhi = 1; ihi = 0; } else { inhi = 0; ihi = 1; }
      for (int i = 0; i < mpts; i++) {
        if (gv[i] <= gv[ilo]) ilo = i;
        if (gv[i] > gv[ihi]) { inhi = ihi; ihi = i; }
        else if (gv[i] > gv[inhi] && i != ihi) inhi = i;
      }
      const float rtol = (float)(2.0 * (double)fabsf(gv[ihi] - gv[ilo]) /
                                 (double)(fabsf(gv[ihi]) + fabsf(gv[ilo]) + tiny));
      const float rtol_diff = fabsf(rtol - old_rtol);
      old_rtol = rtol;
      if (fabsf(gamma_new - gamma_old) < 1.0e-8f) gamma_repeats++;
      gamma_old = gamma_new;
      if ((double)rtol < P.robust_tol || (double)rtol_diff < P.robust_tol || gamma_repeats > 15) {
        const float g0 = gv[0];
        gv[0] = gv[ilo];
        gv[ilo] = g0;
        for (int i = 0; i < nd; i++) {
          const float t = pts[0][i];
          pts[0][i] = pts[ilo][i];
          pts[ilo][i] = t;
        }
        break;
      }
      auto trial = [&](float fac) -> float {
        const float fac1 = (float)((1.0 - (double)fac) / nd);
        const float fac2 = fac1 - fac;
        for (int j = 0; j < nd; j++) {
          ptry[j] = psum[j] * fac1 - pts[ihi][j] * fac2;
          vars[j] = ptry[j];
        }
        const float y = evaluate();
        if (y < gv[ihi]) {
          gv[ihi] = y;
          for (int j = 0; j < nd; j++) {
            psum[j] += ptry[j] - pts[ihi][j];
            pts[ihi][j] = ptry[j];
          }
        }
        return y;
      };
      float ytry = trial(-1.0f);
      if (ytry <= gv[ilo]) {
        ytry = trial(2.0f);
      } else if (ytry >= gv[inhi]) {
        const float ysave = gv[ihi];
        ytry = trial(0.5f);
        if (ytry >= ysave) {
          for (int i = 0; i < mpts; i++) {
            if (i != ilo) {
              for (int j = 0; j < nd; j++) {
                pts[i][j] = psum[j] = (float)(0.5 * (double)(pts[i][j] + pts[ilo][j]));
                vars[j] = psum[j];
              }
              gv[i] = evaluate();
            }
          }
          for (int j = 0; j < nd; j++) {
            float sum = 0.0f;
            for (int i = 0; i < mpts; i++) sum += pts[i][j];
            psum[j] = sum;
          }
        }
      }
      gamma_new = evaluate();
    }
    num_iterations = iteration;
    finish();
    return DICEGPU_CORRELATION_SUCCESSFUL;
  }

  // Subset::noise_std_dev (DICe_Subset.cpp:622-703) on the deformed image.
  __device__ float noise_std_dev(const SubsetRef& sb, const PassOut& st, const float* slots) const {
    if (st.n == 0) return -1.0f;
    MapConst k;
    make_mapconst<SHAPE>(slots, false, (float)sb.cx, (float)sb.cy, k);
    float u, v, t;
    map_to_u_v_theta<SHAPE>(k, (float)sb.cx, (float)sb.cy, u, v, t);
    int min_x = (int)((float)st.minx + u), max_x = (int)((float)st.maxx + u);
    int min_y = (int)((float)st.miny + v), max_y = (int)((float)st.maxy + v);
    const int img_w = A.def.w, img_h = A.def.h;
    if (min_x < 0) min_x = 0;
    if (min_y < 0) min_y = 0;
    if (max_x >= img_w) min_x = 0;
    if (max_y >= img_h) min_y = 0;
    int hh = max_y - min_y + 1, ww = max_x - min_x + 1;
    if (ww < 3) ww = 3;
    if (hh < 3) hh = 3;
    const int rw = max_x - min_x, rh = max_y - min_y;
    double acc = 0.0;
    if (rw > 0 && rh > 0) {
      // a lane per column, a sliding 3-row window down the rows; reads go
      // through the row-major linear index like the reference's operator()
      // (0 outside the array), so edge pixels need no special window
      const long lim = (long)img_w * img_h;
      const float* I = A.def.I;
      auto ld = [&](int x, int y) -> float {
        const long li = (long)y * img_w + x;
        return (li >= 0 && li < lim) ? __ldg(I + li) : 0.0f;
      };
      for (int xb = min_x; xb < max_x; xb += 32) {
        const int xx = xb + lane;
        if (xx >= max_x) continue;
        float a0 = ld(xx - 1, min_y - 1), a1 = ld(xx, min_y - 1), a2 = ld(xx + 1, min_y - 1);
        float b0 = ld(xx - 1, min_y), b1 = ld(xx, min_y), b2 = ld(xx + 1, min_y);
        const bool xedge = xx < 1 || xx >= img_w - 1;
        for (int yy = min_y; yy < max_y; ++yy) {
          const float c0 = ld(xx - 1, yy + 1), c1 = ld(xx, yy + 1), c2 = ld(xx + 1, yy + 1);
          if (xedge || yy < 1 || yy >= img_h - 1) {
            acc += (double)fabsf(b1);
          } else {
            // mask[i][j] (i: x offset, j: y offset), j outer, i inner
            float conv = 0.0f;
            conv += a0 * 1.0f;  conv += a1 * -2.0f; conv += a2 * 1.0f;
            conv += b0 * -2.0f; conv += b1 * 4.0f;  conv += b2 * -2.0f;
            conv += c0 * 1.0f;  conv += c1 * -2.0f; conv += c2 * 1.0f;
            acc += (double)fabsf(conv);
          }
          a0 = b0; a1 = b1; a2 = b2;
          b0 = c0; b1 = c1; b2 = c2;
        }
      }
    }
    acc = warp_sum(acc);
    const float var = (float)acc;
    return (float)((double)var * (sqrt(0.5 * 3.14159265358979323846) / (6.0 * (ww - 2) * (hh - 2))));
  }

  // Objective::sigma (DICe_Objective.cpp:150-184)
  __device__ float sigma(const SubsetRef& sb, const PassOut& st, const float* slots, float& noise) const {
    noise = noise_std_dev(sb, st, slots);
    if (noise < 0.0f) return -1.0f;
    const float sgx = (float)st.sgx2, sgy = (float)st.sgy2;
    const float sg = sgx > sgy ? sgy : sgx;
    return sg > 0.0f ? (float)sqrt(2.0 * (double)noise * (double)noise / (double)sg) : -1.0f;
  }

  // initialize_parameters_from_fields from the field row held across the
  // warp (lane c = column c): affine slots 0..5 are DISP_X, DISP_Y, ROT_Z,
  // STRETCH_XX, STRETCH_YY, SHEAR_XY (disabled slots 0); quadratic QUAD_A..L
  __device__ void load_slots_row(double fv, float* slots) const {
    if (SHAPE == DICEGPU_QUADRATIC_SF) {
#pragma unroll
      for (int i = 0; i < 12; ++i) slots[i] = (float)__shfl_sync(FULL, fv, DICEGPU_F_QUAD_A + i);
    } else {
      const unsigned em = enabled_mask();
#pragma unroll
      for (int s = 0; s < 6; ++s) {
        const float v = (float)__shfl_sync(FULL, fv, DICEGPU_F_DISP_X + s);
        slots[s] = ((em >> s) & 1u) ? v : 0.0f;
      }
#pragma unroll
      for (int s = 6; s < 12; ++s) slots[s] = 0.0f;
    }
  }

  // Quadratic_Shape_Function::update_params_for_centroid_change
  // (DICe_LocalShapeFunction.cpp:632-651) for a neighbour's parameters:
  // float parameters and products, the 2.0 literals promote to double.
  __device__ static void centroid_change(float* q, float dx, float dy) {
    const float A = q[0], B = q[1], C = q[2], D = q[3], E = q[4];
    const float G = q[6], H = q[7], I = q[8], J = q[9], K = q[10];
    auto dbl_term = [](float c, float d1, float d, float d2) {   // c*d1 + 2.0*d*d2
      return __dadd_rn((double)__fmul_rn(c, d1), __dmul_rn(__dmul_rn(2.0, (double)d), (double)d2));
    };
    auto flt_sum = [](float a, float b, float c, float d, float e, float dx_, float dy_, float sub) {
      float t = __fadd_rn(__fmul_rn(a, dx_), __fmul_rn(b, dy_));
      t = __fadd_rn(t, __fmul_rn(__fmul_rn(c, dx_), dy_));
      t = __fadd_rn(t, __fmul_rn(__fmul_rn(d, dx_), dx_));
      t = __fadd_rn(t, __fmul_rn(__fmul_rn(e, dy_), dy_));
      return __fsub_rn(t, sub);
    };
    q[0] = (float)__dadd_rn((double)q[0], dbl_term(C, dy, D, dx));
    q[1] = (float)__dadd_rn((double)q[1], dbl_term(C, dx, E, dy));
    q[5] = __fadd_rn(q[5], flt_sum(A, B, C, D, E, dx, dy, dx));
    q[6] = (float)__dadd_rn((double)q[6], dbl_term(I, dy, J, dx));
    q[7] = (float)__dadd_rn((double)q[7], dbl_term(I, dx, K, dy));
    q[11] = __fadd_rn(q[11], flt_sum(G, H, I, J, K, dx, dy, dy));
  }

  // Local_Shape_Function::save_fields: the shape-function columns of a field
  // row from the parameters (quadratic: A..L plus u, v, theta mapped at the
  // subset's coordinates).  Lane 0 writes.
  __device__ void save_shape_fields(double* f, const float* slots, float fcx, float fcy) const {
    if (SHAPE == DICEGPU_QUADRATIC_SF) {
      MapConst k;
      make_mapconst<SHAPE>(slots, false, fcx, fcy, k);
      float u, v, t;
      map_to_u_v_theta<SHAPE>(k, fcx, fcy, u, v, t);
      if (lane == 0) {
        for (int i = 0; i < 12; ++i) f[DICEGPU_F_QUAD_A + i] = slots[i];
        f[DICEGPU_F_DISP_X] = u;
        f[DICEGPU_F_DISP_Y] = v;
        f[DICEGPU_F_ROT_Z] = t;
      }
    } else if (lane == 0) {
      f[DICEGPU_F_DISP_X] = slots[0];
      f[DICEGPU_F_DISP_Y] = slots[1];
      for (int kx = 2; kx < A.P.N; ++kx) f[DICEGPU_F_DISP_X + A.P.slot[kx]] = slots[A.P.slot[kx]];
    }
  }

  // One Objective entry point for a fresh subset at the parameters of its
  // field row (Objective_ZNSSD::computeUpdateFast, DICe_Objective.cpp:430-657;
  // Objective::computeUpdateRobust, :369-388; Objective::sigma after the
  // subset's deformed-state initialisation at those parameters, :150-184).
  // Separate and not inlined so the correlation path keeps its registers.
  __device__ __noinline__ void run_objective(const SubsetRef sb, const double fv) {
    float slots[12];
    load_slots_row(fv, slots);
    double* f = A.fields + (size_t)sb.idx * DICEGPU_FIELD_STRIDE;
    const float fcx = (float)__shfl_sync(FULL, fv, DICEGPU_F_COORD_X);
    const float fcy = (float)__shfl_sync(FULL, fv, DICEGPU_F_COORD_Y);
    if (A.mode == MODE_SIGMA) {
      const PassOut st = pass<false, true, true>(sb, slots, nullptr);
      float noise = 0.0f;
      const float sg = sigma(sb, st, slots, noise);
      if (lane == 0) {
        A.gamma_out[sb.idx] = sg;
        A.noise_out[sb.idx] = noise;
      }
      return;
    }
    int num_iterations = -1;
    int status;
    if (A.mode == MODE_GN) {
      float cond = -1.0f;
      PassOut last;
      status = gauss_newton(sb, slots, 0.0f, true, num_iterations, cond, last);
      if (lane == 0) f[DICEGPU_F_CONDITION] = cond;
    } else {
      float last_eval[12];
      status = simplex(sb, slots, num_iterations, last_eval);
    }
    save_shape_fields(f, slots, fcx, fcy);
    if (lane == 0) {
      A.iter_out[sb.idx] = num_iterations;
      A.status_out[sb.idx] = status;
    }
  }

  __device__ void record_failed(double* f, int status, int num_iterations) const {
    if (lane == 0) {
      f[DICEGPU_F_SIGMA] = -1.0; f[DICEGPU_F_MATCH] = -1.0; f[DICEGPU_F_GAMMA] = -1.0;
      f[DICEGPU_F_BETA] = -1.0; f[DICEGPU_F_OMEGA] = -1.0; f[DICEGPU_F_NOISE] = -1.0;
      f[DICEGPU_F_CONTRAST] = -1.0; f[DICEGPU_F_ACTIVE_PIXELS] = -1.0;
      f[DICEGPU_F_STATUS] = status; f[DICEGPU_F_ITERATIONS] = num_iterations;
    }
  }

  // Objective::beta (DICe_Objective.cpp:78-148)
  __device__ float beta(const SubsetRef& sb, const float* slots) {
    const DevParams& P = A.P;
    MapConst k;
    make_mapconst<SHAPE>(slots, false, (float)sb.cx, (float)sb.cy, k);
    float u0, v0, t0;
    map_to_u_v_theta<SHAPE>(k, (float)sb.cx, (float)sb.cy, u0, v0, t0);
    auto gam = [&](const float* s) {
      PassOut o = pass<false, false, true>(sb, s, nullptr);
      return gamma_from_unnormalised(o);
    };
    const float g0 = gam(slots);
    const float eps = 0.1f;
    const float fac[3] = {1.0e-3f, 1.0e-3f, 1.0e-1f};
    float dir[3] = {0.0f, 0.0f, 0.0f};
    for (int i = 0; i < 3; ++i) {
      if (!P.has_rot && i == 2 && SHAPE != DICEGPU_QUADRATIC_SF) continue;
      if (!P.has_rot && i == 2) continue;
      float u = u0, v = v0, t = t0;
      float s[12];
      auto insert = [&]() {
#pragma unroll
        for (int j = 0; j < 12; ++j) s[j] = slots[j];
        if (SHAPE == DICEGPU_QUADRATIC_SF) {
#pragma unroll
          for (int j = 0; j < 12; ++j) s[j] = 0.0f;
          s[0] = cosf(t); s[1] = -sinf(t); s[6] = sinf(t); s[7] = cosf(t);
          s[5] = u; s[11] = v;
        } else {
          s[0] = u; s[1] = v;
          if (P.has_rot) s[2] = t;
        }
      };
      if (i == 0) u += eps; else if (i == 1) v += eps; else t += eps;
      insert();
      const float gp = gam(s);
      if (i == 0) u -= 2 * eps; else if (i == 1) v -= 2 * eps; else t -= 2 * eps;
      insert();
      const float gm = gam(s);
      if (fabsf(gm - g0) < 1.0e-10f || fabsf(gp - g0) < 1.0e-10f) return -1.0f;
      const float sm = fabsf(eps / (gm - g0)) * fac[i];
      const float sp = fabsf(eps / (gp - g0)) * fac[i];
      dir[i] = (float)((double)(sm + sp) / 2.0);
    }
    float mag = 0.0f;
    for (int i = 0; i < 3; ++i) {
      if (!P.has_rot && i == 2) continue;
      mag += dir[i] * dir[i];
    }
    return sqrtf(mag);
  }

  __device__ float gamma_from_unnormalised(const PassOut& o) const {
    if (o.n == 0) return -1.0f;
    const double n = (double)o.n;
    const double sgg = o.sG2 - o.sG * o.sG / n;
    const double sff = o.sF2 - o.sumF * o.sumF / n;
    const double sgf = o.sGF - o.sG * o.sumF / n;
    if (!(sgg > 0.0) || !(sff > 0.0)) return -1.0f;
    double g = 2.0 - 2.0 * sgf / sqrt(sgg * sff);
    return (float)(g < 0.0 ? 0.0 : g);
  }

  // --------------------------------------------------------------------------
  // generic_correlation_routine for one subset.
  // --------------------------------------------------------------------------
  __device__ void run(int idx) {
    npass_ = 0;
    run_subset(idx);
    if (A.passes_out && lane == 0 && A.mode == MODE_CORRELATE) A.passes_out[idx] = npass_;
  }

  __device__ void run_subset(int idx) {
    const DevParams& P = A.P;
    double* f = A.fields + (size_t)idx * DICEGPU_FIELD_STRIDE;
    // the subset's field row (32 doubles) in one coalesced load: lane c holds
    // column c, read by shuffles
    const double fv = f[lane];
    auto fld = [&](int col) { return __shfl_sync(FULL, fv, col); };
    SubsetRef sb;
    sb.idx = idx;
    sb.cx = (int)fld(DICEGPU_F_COORD_X);
    sb.cy = (int)fld(DICEGPU_F_COORD_Y);
    if (A.geo.half >= 0) {
      const int side = 2 * A.geo.half + 1;
      sb.npix = side * side;
      sb.off = -1;
    } else {
      sb.off = A.geo.offsets[idx];
      sb.npix = A.geo.offsets[idx + 1] - sb.off;
    }
    {
      const int kx = min(max(sb.cx, 0), A.ref.w - 1), ky = min(max(sb.cy, 0), A.ref.h - 1);
      sb.K = __ldg(A.ref.I + (size_t)ky * A.ref.w + kx);
    }
    sb.masked = false;
    sb.evo = false;
    sb.nact = sb.npix;
    if (MASK && A.geo.mask_desc) {
      const int32_t* md = A.geo.mask_desc + (size_t)idx * DG_MASK_DESC;
      sb.evo = md[DG_DESC_EVOLVE] != 0 && A.geo.pix_flag != nullptr && sb.off >= 0;
      if (sb.evo) sb.nact = A.geo.evo_nact[idx];
      sb.masked = md[2] > 0 || md[5] > 0 || sb.evo;
    }

    float slots[12];
    if (A.mode == MODE_GAMMA) {
      load_slots_row(fv, slots);
      const float g = eval_gamma(sb, slots);
      if (lane == 0) A.gamma_out[idx] = g;
      return;
    }
    if (A.mode != MODE_CORRELATE) {
      run_objective(sb, fv);
      return;
    }
    // frame-0 field-of-view test (DICe_Schema.cpp:2036-2048), whenever a
    // subset size is set (subset_dim_ > 0), whatever the subsets' shapes
    if (P.subset_size > 0 && A.first_frame) {
      const float cur_x = (float)(fld(DICEGPU_F_COORD_X) + fld(DICEGPU_F_DISP_X));
      const float cur_y = (float)(fld(DICEGPU_F_COORD_Y) + fld(DICEGPU_F_DISP_Y));
      const int hs = P.subset_size / 2;
      if (cur_x < hs || cur_x > A.def.w - hs || cur_y < hs || cur_y > A.def.h - hs) {
        record_failed(f, DICEGPU_INITIALIZE_FAILED_BY_EXCEPTION, -1);
        return;
      }
    }
    int num_iterations = -1;
    // Field_Value_Initializer::initial_guess (DICe_Initializer.cpp:398-436):
    // the subset's own row, or its neighbour's.  Subsets run in index order
    // in the reference: a lower neighbour ran earlier this frame (an earlier
    // wave, or this warp just before in a chain: __syncwarp orders lane 0's
    // writes), a higher one contributes its frame-start row.
    double gv = fv;
    int init_status = DICEGPU_INITIALIZE_USING_PREVIOUS_FRAME_SUCCESSFUL;
    const int nb = A.neigh ? A.neigh[idx] : -1;
    if (nb >= 0 && nb < A.n && nb != idx) {
      __syncwarp();
      gv = (nb < idx ? A.fields : A.nsnap)[(size_t)nb * DICEGPU_FIELD_STRIDE + lane];
      init_status = DICEGPU_INITIALIZE_USING_NEIGHBOR_VALUE_SUCCESSFUL;
    }
    if (__shfl_sync(FULL, gv, DICEGPU_F_SIGMA) == -1.0) {
      record_failed(f, DICEGPU_INITIALIZE_FAILED, num_iterations);
      return;
    }
    // the guess is rebuilt from its row for the fallback optimizer (a
    // second initial_guess call in the reference) rather than kept in registers
    const int guess_status = init_status;
    auto initial_guess = [&]() {
      load_slots_row(gv, slots);
      if (SHAPE == DICEGPU_QUADRATIC_SF && guess_status == DICEGPU_INITIALIZE_USING_NEIGHBOR_VALUE_SUCCESSFUL)
        centroid_change(slots,
                        __fsub_rn((float)fld(DICEGPU_F_COORD_X), (float)__shfl_sync(FULL, gv, DICEGPU_F_COORD_X)),
                        __fsub_rn((float)fld(DICEGPU_F_COORD_Y), (float)__shfl_sync(FULL, gv, DICEGPU_F_COORD_Y)));
    };
    initial_guess();
    // reference mean at Gauss-Newton entry: over the pixels active at the last
    // deformed-state initialisation (none yet: all of them)
    bool have_state = false;
    PassOut last_state;
    float last_eval[12];
    if (P.init_gamma_thr != -1.0) {
      PassOut o;
      const float g0 = eval_gamma(sb, slots, &o);
      have_state = true;
      last_state = o;
      if (g0 > P.init_gamma_thr || g0 < 0.0f) {
        record_failed(f, DICEGPU_INITIALIZE_FAILED, num_iterations);
        return;
      }
    }
    const float prev_u = (float)fld(DICEGPU_F_DISP_X);
    const float prev_v = (float)fld(DICEGPU_F_DISP_Y);
    const float prev_t = (float)fld(DICEGPU_F_ROT_Z);
    const bool force_simplex = A.geo.force_simplex && A.geo.force_simplex[idx];
    const int opt = P.opt;
    int corr_status = DICEGPU_CORRELATION_FAILED;
    float cond = 0.0f;
    bool cond_set = false;
    bool state_from_simplex = false;
    (void)state_from_simplex;
    auto run_gn = [&]() {
      // Subset::mean(REF_INTENSITIES) at entry: over the pixels active at the
      // last deformed-state initialisation, or all pixels of a fresh subset
      // (then taken from the first pass)
      float meanF = 0.0f;
      if (have_state) {
        const int n = last_state.n;
        meanF = n ? (float)((last_state.sumF + (double)n * (double)sb.K) / (double)n) : 0.0f;
      }
      corr_status = gauss_newton(sb, slots, meanF, !have_state, num_iterations, cond, last_state);
      have_state = true;
      state_from_simplex = false;
      cond_set = true;
    };
    auto run_simplex = [&]() {
      corr_status = simplex(sb, slots, num_iterations, last_eval);
      // state of the last evaluation: active set, gradients and bounding box
      last_state = pass<false, true, true>(sb, last_eval, nullptr);
      ++npass_;
      have_state = true;
      state_from_simplex = true;
    };
    DG_PT(t_first);
    if (opt == DICEGPU_SIMPLEX || opt == DICEGPU_SIMPLEX_THEN_GRADIENT_BASED || force_simplex) {
      run_simplex();
    } else {
      run_gn();
    }
    DG_PACC(2, t_first);
    MapConst kc;
    const float fcx = (float)fld(DICEGPU_F_COORD_X), fcy = (float)fld(DICEGPU_F_COORD_Y);
    float nu, nv, nt;
    make_mapconst<SHAPE>(slots, false, fcx, fcy, kc);
    map_to_u_v_theta<SHAPE>(kc, fcx, fcy, nu, nv, nt);
    bool jump_pass = !(fabsf(nu - prev_u) > P.disp_jump || fabsf(nv - prev_v) > P.disp_jump ||
                       fabsf(nt - prev_t) > P.theta_jump);
    if (corr_status != DICEGPU_CORRELATION_SUCCESSFUL || !jump_pass) {
      bool second_failed = false;
      if (opt == DICEGPU_SIMPLEX || opt == DICEGPU_GRADIENT_BASED || force_simplex) {
        second_failed = true;
      } else if (opt == DICEGPU_GRADIENT_BASED_THEN_SIMPLEX) {
        initial_guess();
        init_status = guess_status;
        run_simplex();
        if (corr_status != DICEGPU_CORRELATION_SUCCESSFUL) second_failed = true;
      } else if (opt == DICEGPU_SIMPLEX_THEN_GRADIENT_BASED) {
        initial_guess();
        init_status = guess_status;
        run_gn();
        if (corr_status != DICEGPU_CORRELATION_SUCCESSFUL) second_failed = true;
      }
      if (second_failed && corr_status != DICEGPU_CORRELATION_SUCCESSFUL) {
        if (cond_set && lane == 0) f[DICEGPU_F_CONDITION] = cond;
        record_failed(f, corr_status, num_iterations);
        return;
      }
      // the second jump test and save_fields map the parameters of the
      // second attempt (DICe_Schema.cpp:2331-2334)
      make_mapconst<SHAPE>(slots, false, fcx, fcy, kc);
      map_to_u_v_theta<SHAPE>(kc, fcx, fcy, nu, nv, nt);
    }
    if (cond_set && lane == 0) f[DICEGPU_F_CONDITION] = cond;
    // sigma needs the gradients of the last deformed-state initialisation
    const PassOut st = last_state;
    float noise = 0.0f;
    DG_PT(t_sig);
    const float sg = sigma(sb, st, slots, noise);
    DG_PACC(3, t_sig);
    if (sg < 0.0f) {
      record_failed(f, DICEGPU_FRAME_FAILED_DUE_TO_NEGATIVE_SIGMA, num_iterations);
      return;
    }
    PassOut fin;
    DG_PT(t_gam);
    const float gamma = eval_gamma(sb, slots, &fin);
    DG_PACC(4, t_gam);
    const float bt = P.output_beta ? beta(sb, slots) : 0.0f;
    if ((P.final_gamma_thr != -1.0 && gamma > P.final_gamma_thr) || gamma < 0.0f) {
      record_failed(f, DICEGPU_FRAME_FAILED_DUE_TO_HIGH_GAMMA, num_iterations);
      return;
    }
    if (fabsf(nu - prev_u) > P.disp_jump || fabsf(nv - prev_v) > P.disp_jump ||
        fabsf(nt - prev_t) > P.theta_jump) {
      record_failed(f, DICEGPU_JUMP_TOLERANCE_EXCEEDED, num_iterations);
      return;
    }
    // contrast_std_dev and num_active_pixels at the final parameters
    float contrast = 0.0f;
    if (fin.n > 0) {
      const double nn = (double)fin.n;
      double sgg = fin.sG2 - fin.sG * fin.sG / nn;
      if (sgg < 0.0) sgg = 0.0;
      contrast = (float)sqrt(sgg / nn);
    }
    if (lane == 0) {
      // record_step (DICe_Schema.cpp:1986-2009), save_fields
      if (SHAPE == DICEGPU_QUADRATIC_SF) {
        for (int i = 0; i < 12; ++i) f[DICEGPU_F_QUAD_A + i] = slots[i];
        f[DICEGPU_F_DISP_X] = nu;
        f[DICEGPU_F_DISP_Y] = nv;
        f[DICEGPU_F_ROT_Z] = nt;
      } else {
        f[DICEGPU_F_DISP_X] = slots[0];
        f[DICEGPU_F_DISP_Y] = slots[1];
        for (int kx = 2; kx < P.N; ++kx) {
          const int s = P.slot[kx];
          f[DICEGPU_F_DISP_X + s] = slots[s];
        }
      }
      f[DICEGPU_F_SIGMA] = sg;
      f[DICEGPU_F_MATCH] = 0.0;
      f[DICEGPU_F_GAMMA] = gamma;
      f[DICEGPU_F_BETA] = bt;
      f[DICEGPU_F_NOISE] = noise;
      f[DICEGPU_F_CONTRAST] = contrast;
      f[DICEGPU_F_ACTIVE_PIXELS] = fin.n;
      f[DICEGPU_F_STATUS] = init_status;
      f[DICEGPU_F_ITERATIONS] = num_iterations;
    }
    if constexpr (MASK) {
      if (sb.evo && A.evolve) {
        Slots fs;
#pragma unroll
        for (int i = 0; i < 12; ++i) fs.s[i] = slots[i];
        evolve(sb, fs);
      }
    }
  }
};

}  // namespace dg
