// dg_adjoint.cuh -- reverse-mode derivative of the subset objective.
//
// For each subset the forward map is the path of the correlation engine:
// warp of the subset pixels by the shape function (affine or quadratic,
// DICe_LocalShapeFunction.cpp:220-248, 509-520), Keys fourth-order
// interpolation of the deformed image (DICe_Image.cpp:834-883) and the
// objective over the active pixels, either
//   objective 0: gamma = sum (G~/|G~| - F~/|F~|)^2 = 2 - 2 S / (|G~| |F~|)
//                (Objective::gamma, DICe_Objective.cpp:58-76, with
//                G~ = G - mean G, F~ = F - mean F, S = sum G~ F~), or
//   objective 1: C = sum (G~ - F~)^2, the least-squares objective whose
//                Gauss-Newton right-hand side q (DICe_Objective.cpp:523-546)
//                is dC/dp / 2.
// Both are functions of G only through dObj/dG_i = a F~_i + b G~_i (the
// derivatives of the means cancel because sum G~ = sum F~ = 0):
//   gamma: a = -2 / (|G~| |F~|), b = 2 S / (|G~|^3 |F~|);   C: a = -2, b = 2.
// One warp per subset, two passes: the moments give the objective and (a, b);
// the second pass forms lambda_i = seed * (a F~_i + b G~_i), accumulates
// dObj/dp = sum lambda_i dG_i/dp (dG/dp = the shape-function Jacobian applied
// to the interpolant's spatial derivative) and scatters lambda_i times the 36
// interpolation weights into dObj/dI for the deformed image.
//
// The spatial derivative is either the exact derivative of the Keys
// interpolant (grad_source 0: what finite differences of the forward map
// measure) or the Keys interpolation of the gradient images (grad_source 1:
// the Gauss-Newton residual's approximation, DICe_LocalShapeFunction.cpp:
// 350-396, which makes dC/dp equal 2 q exactly).  The 4-pixel border
// deactivation (DICe_Subset.cpp:408) is piecewise constant in the
// parameters and contributes no derivative.
#pragma once

#include "dg_device.cuh"

namespace dg {

struct AdjointArgs {
  DevParams P;
  DevImage ref;
  DevImage def;            // I plane; gx / gy planes for grad_source 1
  DevGeometry geo;
  const double* fields;    // n x DICEGPU_FIELD_STRIDE: parameters per subset
  const double* seed;      // dL/dObj per subset (nullptr: 1)
  int n;
  int objective;           // 0 gamma, 1 least squares
  int grad_source;         // 0 interpolant derivative, 1 interpolated gradient images
  double* value_out;       // n objective values (nullptr: skip)
  double* dparams_out;     // n x 12 derivatives in slot order (nullptr: skip)
  float* ddef;             // W x H accumulated derivative (nullptr: skip)
};

// Derivatives of the Keys kernel pieces (DICe_Image.cpp:114-122): for
// s in [0,1) 4 s^2 - 14/3 s; [1,2) -7/4 s^2 + 6 s - 59/12; [2,3) 1/4 s^2 - 4/3 s + 7/4.
__device__ __forceinline__ float dkeys0(float s) { return fmaf(4.0f, s, -14.0f / 3.0f) * s; }
__device__ __forceinline__ float dkeys1(float s) { return fmaf(fmaf(-1.75f, s, 6.0f), s, -59.0f / 12.0f); }
__device__ __forceinline__ float dkeys2(float s) { return fmaf(fmaf(0.25f, s, -4.0f / 3.0f), s, 1.75f); }
// d/dt of keys_weights(t, w)
__device__ __forceinline__ void dkeys_weights(float t, float d[6]) {
  d[0] = dkeys2(t + 2.0f);
  d[1] = dkeys1(t + 1.0f);
  d[2] = dkeys0(t);
  d[3] = -dkeys0(1.0f - t);
  d[4] = -dkeys1(2.0f - t);
  d[5] = -dkeys2(3.0f - t);
}

template <int SHAPE>
__device__ void adjoint_subset(const AdjointArgs& A, int idx) {
  const int lane = threadIdx.x & 31;
  const double* f = A.fields + (size_t)idx * DICEGPU_FIELD_STRIDE;
  const int cx = (int)f[DICEGPU_F_COORD_X], cy = (int)f[DICEGPU_F_COORD_Y];
  const float fcx = (float)cx, fcy = (float)cy;
  float slots[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) slots[i] = 0.0f;
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
#pragma unroll
    for (int i = 0; i < 12; ++i) slots[i] = (float)f[DICEGPU_F_QUAD_A + i];
  } else {
#pragma unroll
    for (int i = 0; i < 6; ++i) slots[i] = (float)f[DICEGPU_F_DISP_X + i];
  }
  MapConst k;
  make_mapconst<SHAPE>(slots, false, fcx, fcy, k);
  int npix, off;
  if (A.geo.half >= 0) {
    const int side = 2 * A.geo.half + 1;
    npix = side * side;
    off = -1;
  } else {
    off = A.geo.offsets[idx];
    npix = A.geo.offsets[idx + 1] - off;
  }
  const int W = A.def.w, H = A.def.h;
  const long rlim = (long)A.ref.w * A.ref.h;
  auto pixel = [&](int p, int& x, int& y) {
    if (off < 0) {
      const int side = 2 * A.geo.half + 1;
      const int row = p / side;
      x = cx - A.geo.half + (p - row * side);
      y = cy - A.geo.half + row;
    } else {
      x = __ldg(A.geo.px + off + p);
      y = __ldg(A.geo.py + off + p);
    }
    x = max(x, 0);
    y = max(y, 0);
  };
  // pass 1: moments over the active pixels
  double n = 0.0, sF = 0.0, sF2 = 0.0, sG = 0.0, sG2 = 0.0, sGF = 0.0;
  for (int p = lane; p < npix; p += 32) {
    int x, y;
    pixel(p, x, y);
    float mx, my, Dx, Dy;
    map_offset<SHAPE>(k, __fsub_rn((float)x, fcx), __fsub_rn((float)y, fcy), fcx, fcy, mx, my, Dx, Dy);
    const int px = round_pixel(mx), py = round_pixel(my);
    if (px < 4 || px >= W - 4 || py < 4 || py >= H - 4) continue;
    const long ri = (long)y * A.ref.w + x;
    const double F = ri < rlim ? (double)__ldg(A.ref.I + ri) : 0.0;
    float G, gdum, hdum;
    keys_fast_interior<false>(A.def, mx, my, G, gdum, hdum);
    n += 1.0;
    sF += F;
    sF2 += F * F;
    sG += (double)G;
    sG2 += (double)G * (double)G;
    sGF += (double)G * F;
  }
  n = warp_sum(n);
  sF = warp_sum(sF);
  sF2 = warp_sum(sF2);
  sG = warp_sum(sG);
  sG2 = warp_sum(sG2);
  sGF = warp_sum(sGF);
  const double mF = n > 0.0 ? sF / n : 0.0, mG = n > 0.0 ? sG / n : 0.0;
  const double ff = sF2 - n * mF * mF, gg = sG2 - n * mG * mG, S = sGF - n * mG * mF;
  bool valid = n > 0.0;
  double value, a = 0.0, b = 0.0;
  if (A.objective == 0) {
    valid = valid && ff > 0.0 && gg > 0.0;
    const double nf = sqrt(ff), ng = sqrt(gg);
    value = valid ? 2.0 - 2.0 * S / (ng * nf) : -1.0;
    if (valid) {
      a = -2.0 / (ng * nf);
      b = 2.0 * S / (gg * ng * nf);
    }
  } else {
    value = valid ? gg + ff - 2.0 * S : -1.0;
    a = -2.0;
    b = 2.0;
  }
  const double sd = A.seed ? A.seed[idx] : 1.0;
  a *= sd;
  b *= sd;
  double dp[12];
#pragma unroll
  for (int i = 0; i < 12; ++i) dp[i] = 0.0;
  if (valid && (A.dparams_out || A.ddef)) {
    // pass 2: lambda_i, dObj/dp and the scatter into dObj/dI
    for (int p = lane; p < npix; p += 32) {
      int x, y;
      pixel(p, x, y);
      const float dxf = __fsub_rn((float)x, fcx), dyf = __fsub_rn((float)y, fcy);
      float mx, my, Dx, Dy;
      map_offset<SHAPE>(k, dxf, dyf, fcx, fcy, mx, my, Dx, Dy);
      const int px = round_pixel(mx), py = round_pixel(my);
      if (px < 4 || px >= W - 4 || py < 4 || py >= H - 4) continue;
      const long ri = (long)y * A.ref.w + x;
      const double F = ri < rlim ? (double)__ldg(A.ref.I + ri) : 0.0;
      const int ix = (int)mx, iy = (int)my;
      float wx[6], wy[6], dwx[6], dwy[6];
      keys_weights(mx - (float)ix, wx);
      keys_weights(my - (float)iy, wy);
      dkeys_weights(mx - (float)ix, dwx);
      dkeys_weights(my - (float)iy, dwy);
      const size_t base = (size_t)(iy - 2) * W + (ix - 2);
      float G = 0.0f, gx = 0.0f, gy = 0.0f;
#pragma unroll
      for (int m = 0; m < 6; ++m) {
        float rI = 0.0f, rdx = 0.0f, rgx = 0.0f, rgy = 0.0f;
#pragma unroll
        for (int q = 0; q < 6; ++q) {
          const size_t t = base + (size_t)m * W + q;
          const float v = __ldg(A.def.I + t);
          rI = fmaf(wx[q], v, rI);
          if (A.grad_source == 0) {
            rdx = fmaf(dwx[q], v, rdx);
          } else {
            rgx = fmaf(wx[q], __ldg(A.def.gx + t), rgx);
            rgy = fmaf(wx[q], __ldg(A.def.gy + t), rgy);
          }
        }
        G = fmaf(wy[m], rI, G);
        if (A.grad_source == 0) {
          gx = fmaf(wy[m], rdx, gx);
          gy = fmaf(dwy[m], rI, gy);
        } else {
          gx = fmaf(wy[m], rgx, gx);
          gy = fmaf(wy[m], rgy, gy);
        }
      }
      const double lam = a * (F - mF) + b * ((double)G - mG);
      if (A.dparams_out) {
        float r[12];
        residuals_D<SHAPE>(k, dxf, dyf, Dx, Dy, gx, gy, false, r);
        constexpr int NS = SHAPE == DICEGPU_QUADRATIC_SF ? 12 : 6;
#pragma unroll
        for (int i = 0; i < NS; ++i) dp[i] = fma(lam, (double)r[i], dp[i]);
      }
      if (A.ddef) {
        const float lf = (float)lam;
#pragma unroll
        for (int m = 0; m < 6; ++m) {
          const float lm = lf * wy[m];
#pragma unroll
          for (int q = 0; q < 6; ++q) atomicAdd(A.ddef + base + (size_t)m * W + q, lm * wx[q]);
        }
      }
    }
  }
  if (A.dparams_out) {
#pragma unroll
    for (int i = 0; i < 12; ++i) dp[i] = warp_sum(dp[i]);
    if (lane == 0) {
#pragma unroll
      for (int i = 0; i < 12; ++i) A.dparams_out[(size_t)idx * 12 + i] = dp[i];
    }
  }
  if (A.value_out && lane == 0) A.value_out[idx] = value;
}

template <int SHAPE>
__global__ void __launch_bounds__(256) adjoint_kernel(const __grid_constant__ AdjointArgs a) {
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int idx = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; idx < a.n; idx += warps)
    adjoint_subset<SHAPE>(a, idx);
}

}  // namespace dg
