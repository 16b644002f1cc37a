// dg_engine.cuh -- the per-subset correlation engine, one CTA per subset.
//
// Mirrors Schema::generic_correlation_routine (DICe_Schema.cpp:2026-2368)
// with the field-value initializer (the subset's own row, or its
// neighbour's):
//   initial guess -> Gauss-Newton (Objective_ZNSSD::computeUpdateFast,
//   DICe_Objective.cpp:430-657) and/or Nelder-Mead (Simplex::minimize,
//   DICe_Simplex.cpp:60-277) -> jump test -> sigma -> gamma -> record_step.
//
// Every thread of the CTA runs this control code on the same values (the
// parameters, the pass results broadcast through shared memory), so all of
// them take the same branches and meet at the same barriers; the passes
// split the subset's pixels across the CTA (dg_pass.cuh).  The Gauss-Newton
// solve runs in warp 0 and is broadcast; one thread writes the field row.
//
// The arithmetic is the reference's: float where it computes in float, each
// operation rounded on its own (the library is compiled without contraction),
// sums in the reference's order where it sums in float, the FP64 LU factors
// and explicit inverse of LAPACK's DGETRF / DGETRI (unblocked order), and the
// parameter update accumulated in float.
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
  int npix_cap;          // per-pixel array capacity (>= every subset's pixel count)
  unsigned char* pix_scratch;   // per-CTA pixel arrays in global memory (null: shared memory)
  size_t pix_stride;            // bytes per CTA in pix_scratch
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
// border, the 6 x 6 Keys sum (rows outer) elsewhere, in the reference's
// arithmetic.
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
  float iv, a, b;
  keys_ref_interior<false>(im, lx, ly, iv, a, b);
  return iv;
}

struct SubsetRef {
  int idx, cx, cy, npix;
  int off;          // list offset (-1 for squares)
  bool masked;      // has an obstruction bitmap, blocked polygons or evolution state
  bool evo;         // evolving: its list keeps inactive pixels (per-pixel state)
  int nact;         // pixels with is_active set (npix unless evolving)
};

template <int SHAPE, int INTERP, bool DEFGRAD, bool MASK>
struct Engine {
  using L = Layout<SHAPE>;
  const FrameArgs& A;
  const int tid, lane, warp, T;
  int npass_ = 0;   // pixel passes of the current subset (for work accounting)

  __device__ explicit Engine(const FrameArgs& a)
      : A(a), tid(threadIdx.x), lane(threadIdx.x & 31), warp(threadIdx.x >> 5), T(blockDim.x) {}

  __device__ __forceinline__ float* pix() const { return pix_base<SHAPE>(A.pix_scratch, A.pix_stride); }
  __device__ __forceinline__ PixArrays arrays() const { return pix_arrays_at<SHAPE>(pix(), A.npix_cap); }

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

  __device__ __forceinline__ PassInMasked make_in(const SubsetRef& sb) const {
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
    in.cap = A.npix_cap;
    in.pix = pix();
    in.mdesc = nullptr;
    in.mbits = nullptr;
    in.bpoly = nullptr;
    in.bvx = nullptr;
    in.bvy = nullptr;
    in.pflag = nullptr;
    in.pfv = nullptr;
    if (MASK && sb.masked) {
      in.mdesc = A.geo.mask_desc + (size_t)sb.idx * DG_MASK_DESC;
      in.mbits = A.geo.mask_bits;
      in.bpoly = A.geo.blocked_poly;
      in.bvx = A.geo.blocked_vx;
      in.bvy = A.geo.blocked_vy;
      in.pflag = sb.evo ? A.geo.pix_flag : nullptr;
      in.pfv = sb.evo ? A.geo.pix_f : nullptr;
    }
    return in;
  }

  // One pass over the subset at the parameters in `slots` (see cta_pass).
  template <int KIND>
  __device__ __forceinline__ void pass(const SubsetRef& sb, const float* slots) {
    MapConst k;
    make_mapconst<SHAPE>(slots, !DEFGRAD, (float)sb.cx, (float)sb.cy, k);
    const PassInMasked in = make_in(sb);
    if (MASK && sb.masked) {
      cta_pass<SHAPE, INTERP, DEFGRAD, KIND, true>(in, k);
    } else {
      cta_pass<SHAPE, INTERP, DEFGRAD, KIND, false>(static_cast<const PassIn&>(in), k);
    }
    ++npass_;
  }

  // Subset::gamma (DICe_Subset.cpp:323-340) over the live pixels of the last
  // pass: mean and root sum of squares of F and of G, then the sum of
  // squared differences of the normalised intensities, each a float sum in
  // pixel order.  `def_sum2` receives the deformed sum of squares before
  // its root (Subset::contrast_std_dev forms the same sum).  Uses rows 0 and
  // 1 as scratch.
  __device__ float gamma_exact(const SubsetRef& sb, float* def_sum2 = nullptr) {
    const PixArrays X = arrays();
    float* T0 = X.R(0);
    float* T1 = X.R(1);
    const int n = ctl().n;
    const int np = sb.npix;
    float s[2];
    // mean(REF_INTENSITIES), mean(DEF_INTENSITIES) (:285-301) over the live
    // pixels (G is 0 at the others)
    for (int p = tid; p < np; p += T) T0[p] = (X.L[p] & 1) ? X.F[p] : 0.0f;
    chains(2, T0, X.G, nullptr, nullptr, nullptr, 0u, np, s);
    const float mr = n ? __fdiv_rn(s[0], (float)n) : 0.0f;
    const float md = n ? __fdiv_rn(s[1], (float)n) : 0.0f;
    for (int p = tid; p < np; p += T) {
      float a = 0.0f, b = 0.0f;
      if (X.L[p] & 1) {
        const float fa = __fsub_rn(X.F[p], mr), gb = __fsub_rn(X.G[p], md);
        a = __fmul_rn(fa, fa);
        b = __fmul_rn(gb, gb);
      }
      T0[p] = a;
      T1[p] = b;
    }
    chains(2, T0, T1, nullptr, nullptr, nullptr, 0u, np, s);
    if (def_sum2) *def_sum2 = s[1];
    const float sr = __fsqrt_rn(s[0]), sd = __fsqrt_rn(s[1]);
    if (sr == 0.0f || sd == 0.0f) return -1.0f;
    for (int p = tid; p < np; p += T) {
      float t = 0.0f;
      if (X.L[p] & 1) {
        const float val = __fsub_rn(__fdiv_rn(__fsub_rn(X.G[p], md), sd), __fdiv_rn(__fsub_rn(X.F[p], mr), sr));
        t = __fmul_rn(val, val);
      }
      T0[p] = t;
    }
    chains(1, T0, nullptr, nullptr, nullptr, nullptr, 0u, np, s);
    return s[0];
  }

  // Objective::gamma (DICe_Objective.cpp:58-76): initialise, Subset::gamma,
  // optionally divided by the number of active pixels (in double).
  __device__ float eval_gamma(const SubsetRef& sb, const float* slots, bool normalize,
                                         float* def_sum2 = nullptr) {
    pass<PK_GAMMA>(sb, slots);
    float g = gamma_exact(sb, def_sum2);
    if (normalize && sb.nact > 0) g = (float)((double)g / (double)sb.nact);
    return g;
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
  struct Slots {
    float s[12];
  };
  __device__ __noinline__ void write_uncertainty(const SubsetRef sb, const Slots before, const Slots after) {
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
    for (int p = tid; p < sb.npix; p += T) {
      int x, y;
      pixel_xy(sb, p, x, y);
      const long ri = (long)y * A.ref.w + x;
      const bool rin = ri < rlim;
      float gx = rin ? __ldg(A.ref.gx + ri) : 0.0f;
      float gy = rin ? __ldg(A.ref.gy + ri) : 0.0f;
      if (DEFGRAD) {
        float mx, my, Dx, Dy;
        map_offset<SHAPE>(kb, __fsub_rn((float)x, fcx), __fsub_rn((float)y, fcy), fcx, fcy, mx, my, Dx, Dy);
        const int px = round_pixel(mx), py = round_pixel(my);
        if (!(px < 4 || px >= W - 4 || py < 4 || py >= H - 4)) {
          float G;
          interp_ref<INTERP, true>(A.def, mx, my, G, gx, gy);
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
    s_g2 = cta_sum(s_g2);
    s_uhat = cta_sum(s_uhat);
    s_ug = cta_sum(s_ug);
    s_jg = cta_sum(s_jg);
    s_r = cta_sum(s_r);
    if (tid == 0) {
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
    for (int p = tid; p < sb.npix; p += T) {
      uint8_t* st = A.geo.pix_flag + sb.off + p;
      if (*st != 0) continue;
      int x, y;
      pixel_xy(sb, p, x, y);
      float mx, my, Dx, Dy;
      map_offset<SHAPE>(k, __fsub_rn((float)x, fcx), __fsub_rn((float)y, fcy), fcx, fcy, mx, my, Dx, Dy);
      const int px = round_pixel(mx), py = round_pixel(my);
      if (px < 4 || px >= W - 4 || py < 4 || py >= H - 4 || mv.hides(px, py)) continue;
      float G, gx, gy;
      interp_ref<INTERP, false>(A.def, mx, my, G, gx, gy);
      A.geo.pix_f[sb.off + p] = G;
      *st = 2;
      ++on;
    }
    on = cta_sum_i(on);
    if (tid == 0 && on) A.geo.evo_nact[sb.idx] += on;
  }

  __device__ __forceinline__ void uncertainty_hook(const SubsetRef& sb, const float* before, const float* after) {
    Slots b, a;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
      b.s[i] = before[i];
      a.s[i] = after[i];
    }
    write_uncertainty(sb, b, a);
  }

  // --------------------------------------------------------------------------
  // The Gauss-Newton step of one iteration, run by warp 0: the Hessian and
  // right-hand side from the warps' sums (compact parameter order), the LM
  // penalty, the 2x2 condition number (:558-564, float / double as the
  // reference mixes them), LU with partial pivoting and the explicit inverse
  // (the unblocked DGETRF / DGETRI operations, :571, :591), then
  // def_update[i] = sum_j inv[i][j] * (-1.0) * q[j], accumulated in float
  // (:599-601), the momentum term, the float update of the parameters and the
  // convergence test.  A zero pivot leaves the LU factors in place and the
  // reference applies them as the "inverse" (DGETRI returns early).  Results
  // go to Ctl: status (0, or HESSIAN_SINGULAR), cond, conv, slots.
  // --------------------------------------------------------------------------
  // hw0, hnw: the warps whose Hessian sums hold the subset's pixels (h_sweep)
  __device__ __forceinline__ void solve_step(const Slots cur, int hw0, int hnw) {
    const DevParams& P = A.P;
    const int N = P.N;
    Ctl& c = ctl();
    const WarpOut<SHAPE>* wo = wouts<SHAPE>();
    const int NW = T >> 5;
    for (int e = lane; e < N * N; e += 32) {
      const int a = e / N, b = e - a * N;
      const int i = P.slot[a], j = P.slot[b];
      const int lo = min(i, j), hi = max(i, j);
      double m = 0.0, er = 0.0;
      for (int w = hw0; w < hw0 + hnw; ++w) m += wo[w].M[lo * L::VW + hi];
      for (int w = hw0; w < hw0 + hnw; ++w) er += wo[w].E[pair_index(lo, hi, L::NS)];
      c.H[e] = m - er;
    }
    if (lane < N) {
      double qq = 0.0;
      for (int w = 0; w < NW; ++w) qq += wo[w].q[P.slot[lane]];
      c.q[lane] = qq;
    }
    __syncwarp();
    if (lane == 0 && P.lm_alpha > 0.0f) {
      c.H[0] += (double)P.lm_alpha;
      c.H[N + 1] += (double)P.lm_alpha;
    }
    __syncwarp();
    // 2x2 condition number of the displacement block
    float cond = -1.0f;
    {
      const double H00 = c.H[0], H01 = c.H[1], H10 = c.H[N], H11 = c.H[N + 1];
      const float det_h = (float)(H00 * H11 - H10 * H01);
      const double nsq = H00 * H00 + H01 * H01 + H10 * H10 + H11 * H11;
      const float norm_H = (float)sqrt(nsq);
      if (det_h != 0.0f) {
        const float dd = det_h * det_h;
        const float norm_Hi = (float)sqrt((1.0 / (double)dd) * nsq);
        cond = norm_H * norm_Hi;
      }
    }
    if (lane == 0) c.cond = cond;
    if (cond > 1.0e12f) {
      if (lane == 0) c.status = DICEGPU_HESSIAN_SINGULAR;
      return;
    }
    // LU with partial pivoting in place in c.H (the unblocked DGETRF steps:
    // IDAMAX, the row swap, the scaling by the pivot's reciprocal, the rank-1
    // update), then the inverse a column per lane, x = U^-1 L^-1 P e_lane.
    // Rolled loops over shared memory: the solve runs once per iteration on
    // one warp, and a short loop stays in the instruction cache.
    int info = 0;
#pragma unroll 1
    for (int j = 0; j < N; ++j) {
      double best = fabs(c.H[j * N + j]);
      int p = j;
#pragma unroll 1
      for (int i = j + 1; i < N; ++i) {
        const double ai = fabs(c.H[i * N + j]);
        if (ai > best) { best = ai; p = i; }
      }
      const double pv = c.H[p * N + j];
      __syncwarp();
      if (lane == 0) c.piv[j] = p;
      if (pv != 0.0) {
        if (p != j && lane < N) {
          const double t = c.H[j * N + lane];
          c.H[j * N + lane] = c.H[p * N + lane];
          c.H[p * N + lane] = t;
        }
        __syncwarp();
        const double r = 1.0 / pv;
        if (lane > j && lane < N) c.H[lane * N + j] = c.H[lane * N + j] * r;
      } else if (info == 0) {
        info = j + 1;
      }
      __syncwarp();
      const int m = N - 1 - j;
#pragma unroll 1
      for (int e = lane; e < m * m; e += 32) {
        const int i = j + 1 + e / m, kx = j + 1 + (e - (e / m) * m);
        c.H[i * N + kx] = c.H[i * N + kx] - c.H[i * N + j] * c.H[j * N + kx];
      }
      __syncwarp();
    }
    if (info == 0 && lane < N) {
      double* x = ctl_inv<SHAPE>(c) + lane;     // column `lane`, stride N
      int pos = lane;                           // P e_lane is a unit vector
#pragma unroll 1
      for (int j = 0; j < N; ++j) {
        const int pj = c.piv[j];
        if (pos == j) pos = pj;
        else if (pos == pj) pos = j;
      }
#pragma unroll 1
      for (int i = 0; i < N; ++i) x[i * N] = i == pos ? 1.0 : 0.0;
#pragma unroll 1
      for (int i = 1; i < N; ++i) {
        double acc = x[i * N];
#pragma unroll 1
        for (int j = 0; j < i; ++j) acc = acc - c.H[i * N + j] * x[j * N];
        x[i * N] = acc;
      }
#pragma unroll 1
      for (int i = N - 1; i >= 0; --i) {
        double acc = x[i * N];
#pragma unroll 1
        for (int j = i + 1; j < N; ++j) acc = acc - c.H[i * N + j] * x[j * N];
        x[i * N] = acc / c.H[i * N + i];
      }
    }
    __syncwarp();
    bool notc = false;
    float nw = 0.0f;
    if (lane < N) {
      const double* Mrow = info == 0 ? ctl_inv<SHAPE>(c) + lane * N : &c.H[lane * N];
      float du = 0.0f;
      for (int j = 0; j < N; ++j) du = (float)((double)du + (Mrow[j] * (-1.0)) * c.q[j]);
      if (P.momentum != 0.0f) {
        du = du + P.momentum * c.upd_old[lane];
        c.upd_old[lane] = du;
      }
      // the lane's parameter slot, selected without indexing the register array
      const int sl = P.slot[lane];
      float old = 0.0f;
#pragma unroll
      for (int i = 0; i < 12; ++i)
        if (i == sl) old = cur.s[i];
      nw = old + du;
      // test_for_convergence: affine u, v, theta (DICe_LocalShapeFunction.cpp:433-459),
      // quadratic every parameter (:91-102)
      const bool tested = SHAPE == DICEGPU_QUADRATIC_SF || lane < 2 || (lane == 2 && P.has_rot);
      notc = tested && fabsf(nw - old) >= P.fast_tol;
    }
    const bool conv = !__any_sync(FULL, notc);
    if (lane < 12) c.slots[lane] = cur.s[lane];
    __syncwarp();
    if (lane < N) c.slots[P.slot[lane]] = nw;
    if (lane == 0) {
      c.status = DICEGPU_CORRELATION_SUCCESSFUL;
      c.conv = conv ? 1 : 0;
    }
  }

  // --------------------------------------------------------------------------
  // Gauss-Newton (Objective_ZNSSD::computeUpdateFast).  `slots` in/out.
  // The reference mean at entry (Subset::mean(REF_INTENSITIES), :465) is
  // over the pixels live at the last deformed-state initialisation when
  // `have_state`, else over all active pixels of the fresh subset.
  // --------------------------------------------------------------------------
  __device__ int gauss_newton(const SubsetRef& sb, float* slots, bool have_state, int& num_iterations,
                              float& cond_out) {
    const DevParams& P = A.P;
    Ctl& c = ctl();
    const PixArrays X = arrays();
    float meanF = 0.0f;
    if (have_state) {
      const int na = c.n;
      float s;
      chains(1, X.F, nullptr, nullptr, nullptr, X.L, 0x01u, sb.npix, &s);
      meanF = na ? __fdiv_rn(s, (float)na) : 0.0f;
    }
    if (tid < 12) c.upd_old[tid] = 0.0f;
    int solve_it = 0;
    for (; solve_it <= P.max_fast; ++solve_it) {
      num_iterations = solve_it;
      DG_PT(t_pass);
      pass<PK_GN>(sb, slots);
      DG_PACC(1, t_pass);
      const int n = c.n;
      MapConst k;
      make_mapconst<SHAPE>(slots, !DEFGRAD, (float)sb.cx, (float)sb.cy, k);
      const PassInMasked in = make_in(sb);
      const PassIn& inb = static_cast<const PassIn&>(in);
      const bool fresh = solve_it == 0 && !have_state;
      // Subset::mean(DEF_INTENSITIES) (and for a fresh subset the entry mean
      // of its active reference intensities) in warp 0 while the other warps
      // sweep the Hessian, which does not need it
      const int NW = T >> 5;
      const int hw0 = NW > 1 ? 1 : 0, hnw = NW > 1 ? NW - 1 : 1;
      DG_PT(t_h);
      if (warp == 0 && lane < (fresh ? 2 : 1)) {
        // G is 0 at the pixels that are not live, and every pixel of a subset
        // without evolution state is active
        c.fres[lane] = sb.evo ? chain_sum_masked(lane ? X.F : X.G, X.L, lane ? 2u : 1u, sb.npix)
                              : chain_sum(lane ? X.F : X.G, sb.npix);
      }
      __syncwarp();
      h_sweep<SHAPE, DEFGRAD>(inb, k, hw0, hnw);
      __syncthreads();
      DG_PACC(5, t_h);
      if (fresh) meanF = sb.nact ? __fdiv_rn(c.fres[1], (float)sb.nact) : 0.0f;
      const float meanG = n ? __fdiv_rn(c.fres[0], (float)n) : 0.0f;
      DG_PT(t_q);
      q_sweep<SHAPE, DEFGRAD>(inb, k, meanG, meanF, tid, T);
      __syncthreads();
      DG_PACC(6, t_q);
      Slots cur;
#pragma unroll
      for (int i = 0; i < 12; ++i) cur.s[i] = slots[i];
      DG_PT(t_s);
      if (warp == 0) solve_step(cur, hw0, hnw);
      __syncthreads();
      DG_PACC(7, t_s);
      cond_out = c.cond;
      if (c.status == DICEGPU_HESSIAN_SINGULAR) {
        __syncthreads();
        return DICEGPU_HESSIAN_SINGULAR;
      }
      const bool conv = c.conv != 0;
#pragma unroll
      for (int i = 0; i < 12; ++i) slots[i] = c.slots[i];
      __syncthreads();
      if (conv) {
        if (A.unc && (A.mode == MODE_CORRELATE || A.mode == MODE_GN)) uncertainty_hook(sb, cur.s, slots);
        break;
      }
    }
    if (solve_it > P.max_fast) return DICEGPU_MAX_ITERATIONS_REACHED;
    return DICEGPU_CORRELATION_SUCCESSFUL;
  }

  // --------------------------------------------------------------------------
  // Nelder-Mead (Simplex::minimize, DICe_Simplex.cpp:60-277).  The vertex
  // table and sums live in the warp's SimplexState (lane 0 writes after a
  // __syncwarp, all lanes read after the next); every warp keeps an
  // identical copy and all evaluate the same points together.  `slots`
  // in/out: left at the last evaluated point, as the reference's aliasing
  // of variables and shape-function parameters leaves it
  // (DICe_LocalShapeFunction.h:259-261); `lastp` receives that point in slot
  // form.  The reference evaluates gamma once more at the point it evaluated
  // last before each convergence test; that value is the last one computed,
  // which is taken instead of a second pass.
  // --------------------------------------------------------------------------
  __device__ __forceinline__ void comp_to_slots(const SimplexState& S, const float* comp, float* out) const {
    // out[s] = base[s], then the compact parameters in their slots
#pragma unroll
    for (int s = 0; s < 12; ++s) {
      float v = S.base[s];
#pragma unroll
      for (int kx = 0; kx < 12; ++kx)
        if (kx < A.P.N && A.P.slot[kx] == s) v = comp[kx];
      out[s] = v;
    }
  }

  // Out of line, as beta is: these fallback paths inlined into the
  // correlation loop enlarge the code the Gauss-Newton iterations run
  // through (instruction-cache misses) and slow every subset.
  __device__ __noinline__ int simplex(const SubsetRef& sb, float* slots, int& num_iterations, float* lastp) {
    const DevParams& P = A.P;
    const int nd = P.N;
    const int mpts = nd + 1;
    SimplexState& S = sx_state<SHAPE>();
    const bool w0 = lane == 0;
    float init[12];
#pragma unroll
    for (int kx = 0; kx < 12; ++kx) {
      float v = 0.0f;
#pragma unroll
      for (int s = 0; s < 12; ++s)
        if (kx < nd && P.slot[kx] == s) v = slots[s];
      init[kx] = v;
    }
    __syncwarp();
    if (w0) {
#pragma unroll
      for (int s = 0; s < 12; ++s) S.base[s] = slots[s];
#pragma unroll
      for (int kx = 0; kx < 12; ++kx) S.init[kx] = init[kx];
    }
    __syncwarp();
    float cur[12];   // the last evaluated point (compact)
#pragma unroll
    for (int kx = 0; kx < 12; ++kx) cur[kx] = init[kx];
    float last_y = 0.0f;
    auto evaluate = [&](const float* comp) -> float {
#pragma unroll
      for (int kx = 0; kx < 12; ++kx) cur[kx] = comp[kx];
      comp_to_slots(S, comp, lastp);
      last_y = eval_gamma(sb, lastp, P.normalize_gamma != 0);
      return last_y;
    };
    auto finish = [&]() { comp_to_slots(S, cur, slots); };
    // initial simplex vertex_i = x0 + delta_i e_i (:82-107)
    for (int i = 0; i < mpts; ++i) {
      float v[12];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        v[j] = S.init[j];
        if (i > 0 && j == i - 1) v[j] = v[j] + P.deltas[i - 1];
      }
      __syncwarp();
      if (w0) {
#pragma unroll
        for (int j = 0; j < 12; ++j) S.pts[i][j] = v[j];
      }
      __syncwarp();
      const float g = evaluate(v);
      __syncwarp();
      if (w0) S.gv[i] = g;
      __syncwarp();
      if (i == 0 && g < P.skip_thr && g >= 0.0f) {
        num_iterations = 0;
        finish();
        return DICEGPU_CORRELATION_SUCCESSFUL;
      }
    }
    {
      float ps[12];
#pragma unroll
      for (int j = 0; j < 12; ++j) {
        float sum = 0.0f;
        for (int i = 0; i < mpts; ++i) sum += S.pts[i][j];
        ps[j] = sum;
      }
      __syncwarp();
      if (w0) {
#pragma unroll
        for (int j = 0; j < 12; ++j) S.psum[j] = ps[j];
      }
      __syncwarp();
    }
    int inhi = 0;
    float old_rtol = 0.0f, gamma_new = 0.0f, gamma_old = -1.0f;
    int gamma_repeats = 0;
    const float tiny = 1.0e-10f;
    int ihi = 0;
    // a trial point psum * fac1 - pts[ihi] * fac2 (Simplex::amotry, :188-203),
    // which replaces the worst vertex when it is better
    auto trial = [&](float fac) -> float {
      const float fac1 = (float)((1.0 - (double)fac) / nd);
      const float fac2 = fac1 - fac;
      float pt[12];
#pragma unroll
      for (int j = 0; j < 12; ++j) pt[j] = j < nd ? S.psum[j] * fac1 - S.pts[ihi][j] * fac2 : 0.0f;
      const float y = evaluate(pt);
      if (y < S.gv[ihi]) {
        float ps[12];
#pragma unroll
        for (int j = 0; j < 12; ++j) ps[j] = S.psum[j] + (pt[j] - S.pts[ihi][j]);
        __syncwarp();
        if (w0) {
          S.gv[ihi] = y;
#pragma unroll
          for (int j = 0; j < 12; ++j) {
            if (j < nd) {
              S.psum[j] = ps[j];
              S.pts[ihi][j] = pt[j];
            }
          }
        }
        __syncwarp();
      }
      return y;
    };
    int iteration = 0;
    for (iteration = 0; iteration < P.max_robust; iteration++) {
      if (iteration >= P.max_robust - 1) {
        num_iterations = iteration;
        finish();
        return DICEGPU_MAX_ITERATIONS_REACHED;
      }
      int ilo = 0;
      if (S.gv[0] > S.gv[1]) { inhi = 1; ihi = 0; } else { inhi = 0; ihi = 1; }
      for (int i = 0; i < mpts; i++) {
        const float gi = S.gv[i];
        if (gi <= S.gv[ilo]) ilo = i;
        if (gi > S.gv[ihi]) { inhi = ihi; ihi = i; }
        else if (gi > S.gv[inhi] && i != ihi) inhi = i;
      }
      const float ghi = S.gv[ihi], glo = S.gv[ilo];
      const float rtol = (float)(2.0 * (double)fabsf(ghi - glo) / (double)(fabsf(ghi) + fabsf(glo) + tiny));
      const float rtol_diff = fabsf(rtol - old_rtol);
      old_rtol = rtol;
      if (fabsf(gamma_new - gamma_old) < 1.0e-8f) gamma_repeats++;
      gamma_old = gamma_new;
      if ((double)rtol < P.robust_tol || (double)rtol_diff < P.robust_tol || gamma_repeats > 15) break;
      float ytry = trial(-1.0f);
      if (ytry <= S.gv[ilo]) {
        ytry = trial(2.0f);
      } else if (ytry >= S.gv[inhi]) {
        const float ysave = S.gv[ihi];
        ytry = trial(0.5f);
        if (ytry >= ysave) {
          for (int i = 0; i < mpts; i++) {
            if (i != ilo) {
              float v[12];
#pragma unroll
              for (int j = 0; j < 12; ++j) v[j] = j < nd ? (float)(0.5 * (double)(S.pts[i][j] + S.pts[ilo][j])) : 0.0f;
              __syncwarp();
              if (w0) {
#pragma unroll
                for (int j = 0; j < 12; ++j) {
                  if (j < nd) {
                    S.pts[i][j] = v[j];
                    S.psum[j] = v[j];
                  }
                }
              }
              __syncwarp();
              const float g = evaluate(v);
              __syncwarp();
              if (w0) S.gv[i] = g;
              __syncwarp();
            }
          }
          float ps[12];
#pragma unroll
          for (int j = 0; j < 12; ++j) {
            float sum = 0.0f;
            for (int i = 0; i < mpts; i++) sum += S.pts[i][j];
            ps[j] = sum;
          }
          __syncwarp();
          if (w0) {
#pragma unroll
            for (int j = 0; j < 12; ++j) S.psum[j] = ps[j];
          }
          __syncwarp();
        }
      }
      gamma_new = last_y;
    }
    num_iterations = iteration;
    finish();
    return DICEGPU_CORRELATION_SUCCESSFUL;
  }

  // Subset::noise_std_dev (DICe_Subset.cpp:622-703) on the deformed image
  // over the box of the last pass's live pixels moved by (u, v): the 3 x 3
  // Immerkaer mask (j outer, i inner), |.| summed in float, row by row.  The
  // terms are computed by the CTA a chunk at a time and summed in order by
  // one thread.  Reads go through the row-major linear index like the
  // reference's operator() (0 outside the array).
  struct NoiseBox {
    int min_x, min_y, rw, rh, ww, hh;
    __device__ long total() const { return (rw > 0 && rh > 0) ? (long)rw * rh : 0; }
  };
  __device__ NoiseBox noise_box(const SubsetRef& sb, const float* slots, int bminx, int bmaxx, int bminy,
                                int bmaxy) const {
    MapConst k;
    make_mapconst<SHAPE>(slots, false, (float)sb.cx, (float)sb.cy, k);
    float u, v, t;
    map_to_u_v_theta<SHAPE>(k, (float)sb.cx, (float)sb.cy, u, v, t);
    int min_x = (int)((float)bminx + u), max_x = (int)((float)bmaxx + u);
    int min_y = (int)((float)bminy + v), max_y = (int)((float)bmaxy + v);
    const int img_w = A.def.w, img_h = A.def.h;
    if (min_x < 0) min_x = 0;
    if (min_y < 0) min_y = 0;
    if (max_x >= img_w) min_x = 0;
    if (max_y >= img_h) min_y = 0;
    NoiseBox nb;
    nb.hh = max(max_y - min_y + 1, 3);
    nb.ww = max(max_x - min_x + 1, 3);
    nb.min_x = min_x;
    nb.min_y = min_y;
    nb.rw = max_x - min_x;
    nb.rh = max_y - min_y;
    return nb;
  }
  // The term of box element `id` (row-major over rw x rh).
  __device__ float noise_term(const NoiseBox& nb, long id) const {
    const int img_w = A.def.w, img_h = A.def.h;
    const float* I = A.def.I;
    const int yy = nb.min_y + (int)(id / nb.rw), xx = nb.min_x + (int)(id % nb.rw);
    if (xx < 1 || xx >= img_w - 1 || yy < 1 || yy >= img_h - 1) {
      const long li = (long)yy * img_w + xx;
      const float a = (li >= 0 && li < (long)img_w * img_h) ? __ldg(I + li) : 0.0f;
      return __fsqrt_rn(a * a);
    }
    // mask[i][j] = {{1,-2,1},{-2,4,-2},{1,-2,1}}, i: x offset, j: y offset
    const float* q = I + (size_t)(yy - 1) * img_w + (xx - 1);
    float conv = 0.0f;
    conv = conv + __ldg(q) * 1.0f;
    conv = conv + __ldg(q + 1) * -2.0f;
    conv = conv + __ldg(q + 2) * 1.0f;
    q += img_w;
    conv = conv + __ldg(q) * -2.0f;
    conv = conv + __ldg(q + 1) * 4.0f;
    conv = conv + __ldg(q + 2) * -2.0f;
    q += img_w;
    conv = conv + __ldg(q) * 1.0f;
    conv = conv + __ldg(q + 1) * -2.0f;
    conv = conv + __ldg(q + 2) * 1.0f;
    return fabsf(conv);
  }
  __device__ static float noise_scale(const NoiseBox& nb, float variance) {
    return (float)((double)variance * (sqrt(0.5 * 3.14159265358979323846) / (6.0 * (nb.ww - 2) * (nb.hh - 2))));
  }
  __device__ float noise_exact(const SubsetRef& sb, const float* slots, int n, int bminx, int bmaxx, int bminy,
                               int bmaxy) {
    if (n == 0) return -1.0f;
    const NoiseBox nb = noise_box(sb, slots, bminx, bmaxx, bminy, bmaxy);
    float variance = 0.0f;
    const long total = nb.total();
    const int chunk = A.npix_cap;
    float* buf = arrays().R(0);
    Ctl& c = ctl();
    for (long b0 = 0; b0 < total; b0 += chunk) {
      const int m = (int)min((long)chunk, total - b0);
      for (int e = tid; e < m; e += T) buf[e] = noise_term(nb, b0 + e);
      __syncthreads();
      if (tid == 0) c.fres[0] = chain_sum(buf, m, variance);
      __syncthreads();
      variance = c.fres[0];
      __syncthreads();
    }
    return noise_scale(nb, variance);
  }

  // Objective::sigma (DICe_Objective.cpp:150-184) at the state of the last
  // pass with gradients: noise_std_dev, then the float sums of the squared
  // gradients over the live pixels (the deformed-image gradients stored in
  // rows 0 and 1, or the reference image's at the pixel).
  __device__ float sigma(const SubsetRef& sb, const float* slots, float& noise) {
    Ctl& c = ctl();
    const int n = c.n, bx0 = c.minx, bx1 = c.maxx, by0 = c.miny, by1 = c.maxy;
    const PixArrays X = arrays();
    float* T0 = X.R(0);
    float* T1 = X.R(1);
    const long rlim = (long)A.ref.w * A.ref.h;
    for (int p = tid; p < sb.npix; p += T) {
      float a = 0.0f, b = 0.0f;
      if (X.L[p] & 1) {
        float gx, gy;
        if (DEFGRAD) {
          gx = T0[p];
          gy = T1[p];
        } else {
          int x, y;
          pixel_xy(sb, p, x, y);
          const long ri = (long)y * A.ref.w + x;
          gx = ri < rlim ? __ldg(A.ref.gx + ri) : 0.0f;
          gy = ri < rlim ? __ldg(A.ref.gy + ri) : 0.0f;
        }
        a = gx * gx;
        b = gy * gy;
      }
      T0[p] = a;
      T1[p] = b;
    }
    float s[2];
    const NoiseBox nb = noise_box(sb, slots, bx0, bx1, by0, by1);
    if (PixRows<SHAPE>::NR >= 3 && n > 0 && nb.total() <= A.npix_cap) {
      // the noise terms in row 2, and the three sums side by side
      float* T2 = X.R(2);
      const int nt = (int)nb.total();
      for (int e = tid; e < nt; e += T) T2[e] = noise_term(nb, e);
      Ctl& cl = ctl();
      __syncthreads();
      if (tid < 3) cl.fres[tid] = chain_sum(tid == 0 ? T0 : tid == 1 ? T1 : T2, tid == 2 ? nt : sb.npix);
      __syncthreads();
      s[0] = cl.fres[0];
      s[1] = cl.fres[1];
      noise = noise_scale(nb, cl.fres[2]);
      __syncthreads();
    } else {
      chains(2, T0, T1, nullptr, nullptr, nullptr, 0u, sb.npix, s);
      noise = noise_exact(sb, slots, n, bx0, bx1, by0, by1);
    }
    if (noise < 0.0f) return -1.0f;
    const float sg = s[0] > s[1] ? s[1] : s[0];
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
  // subset's coordinates).  Thread 0 writes.
  __device__ void save_shape_fields(double* f, const float* slots, float fcx, float fcy) const {
    if (SHAPE == DICEGPU_QUADRATIC_SF) {
      MapConst k;
      make_mapconst<SHAPE>(slots, false, fcx, fcy, k);
      float u, v, t;
      map_to_u_v_theta<SHAPE>(k, fcx, fcy, u, v, t);
      if (tid == 0) {
        for (int i = 0; i < 12; ++i) f[DICEGPU_F_QUAD_A + i] = slots[i];
        f[DICEGPU_F_DISP_X] = u;
        f[DICEGPU_F_DISP_Y] = v;
        f[DICEGPU_F_ROT_Z] = t;
      }
    } else if (tid == 0) {
      const unsigned em = enabled_mask();
      f[DICEGPU_F_DISP_X] = slots[0];
      f[DICEGPU_F_DISP_Y] = slots[1];
#pragma unroll
      for (int s = 2; s < 6; ++s)
        if ((em >> s) & 1u) f[DICEGPU_F_DISP_X + s] = slots[s];
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
      pass<PK_STATE>(sb, slots);
      float noise = 0.0f;
      const float sg = sigma(sb, slots, noise);
      if (tid == 0) {
        A.gamma_out[sb.idx] = sg;
        A.noise_out[sb.idx] = noise;
      }
      return;
    }
    int num_iterations = -1;
    int status;
    if (A.mode == MODE_GN) {
      float cond = -1.0f;
      status = gauss_newton(sb, slots, false, num_iterations, cond);
      if (tid == 0) f[DICEGPU_F_CONDITION] = cond;
    } else {
      float last_eval[12];
      status = simplex(sb, slots, num_iterations, last_eval);
    }
    save_shape_fields(f, slots, fcx, fcy);
    if (tid == 0) {
      A.iter_out[sb.idx] = num_iterations;
      A.status_out[sb.idx] = status;
    }
  }

  __device__ void record_failed(double* f, int status, int num_iterations) const {
    if (tid == 0) {
      f[DICEGPU_F_SIGMA] = -1.0; f[DICEGPU_F_MATCH] = -1.0; f[DICEGPU_F_GAMMA] = -1.0;
      f[DICEGPU_F_BETA] = -1.0; f[DICEGPU_F_OMEGA] = -1.0; f[DICEGPU_F_NOISE] = -1.0;
      f[DICEGPU_F_CONTRAST] = -1.0; f[DICEGPU_F_ACTIVE_PIXELS] = -1.0;
      f[DICEGPU_F_STATUS] = status; f[DICEGPU_F_ITERATIONS] = num_iterations;
    }
  }

  // Objective::beta (DICe_Objective.cpp:78-148): the finite-difference slope
  // of the unnormalised gamma in u, v (and theta with rotation), ending with
  // the subset re-initialised at the solution.
  __device__ __noinline__ float beta(const SubsetRef& sb, const float* slots) {
    const DevParams& P = A.P;
    MapConst k;
    make_mapconst<SHAPE>(slots, false, (float)sb.cx, (float)sb.cy, k);
    float u0, v0, t0;
    map_to_u_v_theta<SHAPE>(k, (float)sb.cx, (float)sb.cy, u0, v0, t0);
    const float g0 = eval_gamma(sb, slots, false);
    const float eps = 0.1f;
    const float fac[3] = {1.0e-3f, 1.0e-3f, 1.0e-1f};
    float dir[3] = {0.0f, 0.0f, 0.0f};
    float result = -1.0f;
    bool bad = false;
    for (int i = 0; i < 3 && !bad; ++i) {
      if (!P.has_rot && i == 2) continue;
      float u = u0, v = v0, t = t0;
      float s[12];
      auto insert = [&]() {
#pragma unroll
        for (int j = 0; j < 12; ++j) s[j] = slots[j];
        if (SHAPE == DICEGPU_QUADRATIC_SF) {
          // Quadratic_Shape_Function::insert_motion: clear, then the rigid motion
#pragma unroll
          for (int j = 0; j < 12; ++j) s[j] = 0.0f;
          s[0] = cos_f(t); s[1] = -sin_f(t); s[6] = sin_f(t); s[7] = cos_f(t);
          s[5] = u; s[11] = v;
        } else {
          s[0] = u; s[1] = v;
          if (P.has_rot) s[2] = t;
        }
      };
      if (i == 0) u += eps; else if (i == 1) v += eps; else t += eps;
      insert();
      const float gp = eval_gamma(sb, s, false);
      if (i == 0) u -= 2 * eps; else if (i == 1) v -= 2 * eps; else t -= 2 * eps;
      insert();
      const float gm = eval_gamma(sb, s, false);
      if ((double)fabsf(gm - g0) < 1.0e-10 || (double)fabsf(gp - g0) < 1.0e-10) {
        bad = true;
        break;
      }
      const float sm = fabsf(eps / (gm - g0)) * fac[i];
      const float sp = fabsf(eps / (gp - g0)) * fac[i];
      dir[i] = (float)((double)(sm + sp) / 2.0);
    }
    if (!bad) {
      float mag = 0.0f;
      for (int i = 0; i < 3; ++i) {
        if (!P.has_rot && i == 2) continue;
        mag += dir[i] * dir[i];
      }
      result = __fsqrt_rn(mag);
    }
    return result;
  }

  // Schema::record_step (DICe_Schema.cpp:1986-2009) with save_fields: the
  // shape-function columns (quadratic: A..L and the mapped u, v, theta) and
  // the solve's results.  Thread 0 writes.
  __device__ void record_step(double* f, const float* slots, float nu, float nv, float nt, float sg, float gamma,
                              float bt, float noise, float contrast, int active, int status, int num_iterations) const {
    if (tid != 0) return;
    if (SHAPE == DICEGPU_QUADRATIC_SF) {
      for (int i = 0; i < 12; ++i) f[DICEGPU_F_QUAD_A + i] = slots[i];
      f[DICEGPU_F_DISP_X] = nu;
      f[DICEGPU_F_DISP_Y] = nv;
      f[DICEGPU_F_ROT_Z] = nt;
    } else {
      const unsigned em = enabled_mask();
      f[DICEGPU_F_DISP_X] = slots[0];
      f[DICEGPU_F_DISP_Y] = slots[1];
#pragma unroll
      for (int s = 2; s < 6; ++s)
        if ((em >> s) & 1u) f[DICEGPU_F_DISP_X + s] = slots[s];
    }
    f[DICEGPU_F_SIGMA] = sg;
    f[DICEGPU_F_MATCH] = 0.0;
    f[DICEGPU_F_GAMMA] = gamma;
    f[DICEGPU_F_BETA] = bt;
    f[DICEGPU_F_NOISE] = noise;
    f[DICEGPU_F_CONTRAST] = contrast;
    f[DICEGPU_F_ACTIVE_PIXELS] = active;
    f[DICEGPU_F_STATUS] = status;
    f[DICEGPU_F_ITERATIONS] = num_iterations;
  }

  // The per-pixel state of a subset as constructed (before any deformed-state
  // initialisation): liveness = activity, the rows 0 and 1 = the reference
  // image's gradients at the pixels, live count and box of the active pixels.
  __device__ void fresh_state(const SubsetRef& sb) {
    const PixArrays X = arrays();
    const long rlim = (long)A.ref.w * A.ref.h;
    int n = 0, minx = sb.cx, maxx = sb.cx, miny = sb.cy, maxy = sb.cy;
    for (int p = tid; p < sb.npix; p += T) {
      int x, y;
      pixel_xy(sb, p, x, y);
      bool active = true;
      if (MASK && sb.evo) active = A.geo.pix_flag[sb.off + p] != 0;
      const long ri = (long)y * A.ref.w + x;
      X.R(0)[p] = ri < rlim ? __ldg(A.ref.gx + ri) : 0.0f;
      X.R(1)[p] = ri < rlim ? __ldg(A.ref.gy + ri) : 0.0f;
      X.L[p] = (uint8_t)(active ? 3 : 0);
      if (active) {
        ++n;
        minx = min(minx, x); maxx = max(maxx, x);
        miny = min(miny, y); maxy = max(maxy, y);
      }
    }
    WarpOut<SHAPE>& wo = wouts<SHAPE>()[warp];
    n = warp_sum_i(n);
    minx = warp_min_i(minx); maxx = warp_max_i(maxx);
    miny = warp_min_i(miny); maxy = warp_max_i(maxy);
    if (lane == 0) {
      wo.n = n; wo.minx = minx; wo.maxx = maxx; wo.miny = miny; wo.maxy = maxy;
    }
    __syncthreads();
    if (tid == 0) {
      Ctl& cl = ctl();
      const WarpOut<SHAPE>* all = wouts<SHAPE>();
      int nn = 0, a0 = sb.cx, a1 = sb.cx, b0 = sb.cy, b1 = sb.cy;
      for (int w = 0; w < (T >> 5); ++w) {
        nn += all[w].n;
        a0 = min(a0, all[w].minx); a1 = max(a1, all[w].maxx);
        b0 = min(b0, all[w].miny); b1 = max(b1, all[w].maxy);
      }
      cl.n = nn; cl.minx = a0; cl.maxx = a1; cl.miny = b0; cl.maxy = b1;
    }
    __syncthreads();
  }

  // A subset whose solve is skipped (SKIP_SOLVE, skip_all_solves;
  // DICe_Schema.cpp:2118-2143): sigma, gamma, beta, contrast and the active
  // pixels at the initial guess, recorded as FRAME_SKIPPED.  Out of line: a
  // path outside the correlation loop.
  __device__ __noinline__ void skip_solve(const SubsetRef sb, double* f, const Slots init, int num_iterations) {
    const DevParams& P = A.P;
    float slots[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) slots[i] = init.s[i];
    // Objective::sigma reads the subset as constructed: no deformed-state
    // initialisation has run, so every active pixel counts, with the
    // reference image's gradients, and the noise box is the active pixels'
    fresh_state(sb);
    float noise = 0.0f;
    const float sg = sigma(sb, slots, noise);
    float def_sum2 = 0.0f;
    const float gamma = eval_gamma(sb, slots, P.normalize_gamma != 0, &def_sum2);
    const int fin_n = ctl().n;
    const float bt = P.output_beta ? beta(sb, slots) : 0.0f;
    const float contrast = fin_n == 0 ? 0.0f : __fsqrt_rn(__fdiv_rn(def_sum2, (float)fin_n));
    MapConst kc;
    float nu = 0.0f, nv = 0.0f, nt = 0.0f;
    make_mapconst<SHAPE>(slots, false, (float)sb.cx, (float)sb.cy, kc);
    map_to_u_v_theta<SHAPE>(kc, (float)sb.cx, (float)sb.cy, nu, nv, nt);
    record_step(f, slots, nu, nv, nt, sg, gamma, bt, noise, contrast, fin_n, DICEGPU_FRAME_SKIPPED, num_iterations);
    if constexpr (MASK) {
      if (sb.evo && A.evolve) evolve(sb, init);
    }
  }

  // --------------------------------------------------------------------------
  // generic_correlation_routine for one subset.
  // --------------------------------------------------------------------------
  __device__ void run(int idx) {
    npass_ = 0;
    run_subset(idx);
    if (A.passes_out && tid == 0 && A.mode == MODE_CORRELATE) A.passes_out[idx] = npass_;
  }

  __device__ __noinline__ void run_subset(int idx) {
    const DevParams& P = A.P;
    double* f = A.fields + (size_t)idx * DICEGPU_FIELD_STRIDE;
    // the subset's field row (32 doubles) in one coalesced load per warp:
    // lane c holds column c, read by shuffles
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
      const float g = eval_gamma(sb, slots, P.normalize_gamma != 0);
      if (tid == 0) A.gamma_out[idx] = g;
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
    // wave, or this CTA just before in a chain: the barriers at the end of
    // the previous subset order thread 0's writes), a higher one contributes
    // its frame-start row.
    double gv = fv;
    int init_status = DICEGPU_INITIALIZE_USING_PREVIOUS_FRAME_SUCCESSFUL;
    const int nb = A.neigh ? A.neigh[idx] : -1;
    if (nb >= 0 && nb < A.n && nb != idx) {
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
    const uint8_t subset_flags = A.geo.force_simplex ? A.geo.force_simplex[idx] : 0;
    if ((subset_flags & 2u) || P.skip_all) {
      Slots init;
#pragma unroll
      for (int i = 0; i < 12; ++i) init.s[i] = slots[i];
      skip_solve(sb, f, init, num_iterations);
      return;
    }
    // the deformed state of the subset: none yet (Gauss-Newton then takes the
    // reference mean over all its pixels)
    bool have_state = false;
    float last_eval[12];
    if (P.init_gamma_thr != -1.0) {
      const float g0 = eval_gamma(sb, slots, P.normalize_gamma != 0);
      have_state = true;
      if (g0 > P.init_gamma_thr || g0 < 0.0f) {
        record_failed(f, DICEGPU_INITIALIZE_FAILED, num_iterations);
        return;
      }
    }
    const float prev_u = (float)fld(DICEGPU_F_DISP_X);
    const float prev_v = (float)fld(DICEGPU_F_DISP_Y);
    const float prev_t = (float)fld(DICEGPU_F_ROT_Z);
    const bool force_simplex = (subset_flags & 1u) != 0;
    const int opt = P.opt;
    int corr_status = DICEGPU_CORRELATION_FAILED;
    float cond = 0.0f;
    bool cond_set = false;
    auto run_gn = [&]() {
      corr_status = gauss_newton(sb, slots, have_state, num_iterations, cond);
      have_state = true;
      cond_set = true;
    };
    auto run_simplex = [&]() {
      corr_status = simplex(sb, slots, num_iterations, last_eval);
      // state of the last evaluation: active set, gradients and bounding box
      pass<PK_STATE>(sb, last_eval);
      have_state = true;
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
        if (cond_set && tid == 0) f[DICEGPU_F_CONDITION] = cond;
        record_failed(f, corr_status, num_iterations);
        return;
      }
      // the second jump test and save_fields map the parameters of the
      // second attempt (DICe_Schema.cpp:2331-2334)
      make_mapconst<SHAPE>(slots, false, fcx, fcy, kc);
      map_to_u_v_theta<SHAPE>(kc, fcx, fcy, nu, nv, nt);
    }
    if (cond_set && tid == 0) f[DICEGPU_F_CONDITION] = cond;
    // sigma from the state of the last deformed-state initialisation
    float noise = 0.0f;
    DG_PT(t_sig);
    const float sg = sigma(sb, slots, noise);
    DG_PACC(3, t_sig);
    if (sg < 0.0f) {
      record_failed(f, DICEGPU_FRAME_FAILED_DUE_TO_NEGATIVE_SIGMA, num_iterations);
      return;
    }
    DG_PT(t_gam);
    float def_sum2 = 0.0f;
    const float gamma = eval_gamma(sb, slots, P.normalize_gamma != 0, &def_sum2);
    const int fin_n = ctl().n;
    DG_PACC(4, t_gam);
    // beta ends with the subset re-initialised at the solution, where the
    // gamma pass just left it
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
    // contrast_std_dev (DICe_Subset.cpp:607-620) at the final parameters
    const float contrast = fin_n == 0 ? 0.0f : __fsqrt_rn(__fdiv_rn(def_sum2, (float)fin_n));
    record_step(f, slots, nu, nv, nt, sg, gamma, bt, noise, contrast, fin_n, init_status, num_iterations);
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
