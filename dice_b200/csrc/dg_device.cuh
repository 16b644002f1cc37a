// dg_device.cuh -- device building blocks of the subset-correlation path.
//
// Parameters and images as the kernels see them, warp reductions, the FP64
// tensor-core accumulation, the interpolants (in the reference's arithmetic
// for the correlation path, in a fused FP32 form for the adjoint), the shape
// functions and the pixel rounding of Subset::initialize.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "dicegpu.h"

namespace dg {

constexpr unsigned FULL = 0xffffffffu;

// ---------------------------------------------------------------------------
// Parameters as the kernels see them.
// Affine shape functions are stored in six fixed slots
//   0:u 1:v 2:theta 3:ex 4:ey 5:gxy   (disabled slots stay 0)
// and quadratic ones in twelve slots A..L.  `slot[k]` maps the reference's
// compact parameter index k (spec_map_ insertion order,
// DICe_LocalShapeFunction.cpp:170-218, 461-473) to its slot.
// ---------------------------------------------------------------------------
struct DevParams {
  int shape;       // DICEGPU_AFFINE_SF / DICEGPU_QUADRATIC_SF
  int N;           // number of parameters of the reference shape function
  int NS;          // number of slots (6 affine, 12 quadratic)
  int slot[12];
  int has_rot;
  int interp;
  int opt;
  int max_fast;
  int max_robust;
  float fast_tol;
  double robust_tol;
  float skip_thr;
  float deltas[12];  // simplex deltas, compact order
  double disp_jump;
  double theta_jump;
  float lm_alpha;    // used when > 0
  float momentum;    // used when != 0
  double init_gamma_thr;
  double final_gamma_thr;
  int normalize_gamma;
  int output_beta;
  int use_def_grads;
  int subset_size;
  int skip_all;      // skip_all_solves
};

struct DevImage {
  int w, h;
  const float* __restrict__ I;
  const float* __restrict__ gx;
  const float* __restrict__ gy;
  // (I, Gx, Gy, 0) interleaved: one 16-byte load fetches all three channels
  // of a tap (deformed image with gradients only)
  const float4* __restrict__ p4;
};

// ints per subset mask descriptor: obstruction box (x0, y0, w, h, word
// offset), blocked polygons (count, table offset), subset evolution (1: the
// subset's list keeps its excluded pixels, with per-pixel state), two spare
#define DG_MASK_DESC 10
#define DG_DESC_EVOLVE 7

// Subset geometry: square (`half` >= 0, centred on the COORD fields) or an
// explicit pixel list in CSR form.
struct DevGeometry {
  int half;                       // square half-width, or -1 for lists
  const int32_t* __restrict__ offsets;
  const int32_t* __restrict__ px;
  const int32_t* __restrict__ py;
  const uint8_t* __restrict__ force_simplex;   // per subset: bit 0 force the simplex, bit 1 skip the solve
  // optional per-subset mask descriptors (DG_MASK_DESC ints each), the
  // obstruction words, and the blocked-polygon table and vertices
  const int32_t* __restrict__ mask_desc;
  const uint32_t* __restrict__ mask_bits;
  const int32_t* __restrict__ blocked_poly;
  const int32_t* __restrict__ blocked_vx;
  const int32_t* __restrict__ blocked_vy;
  // subset evolution state of the list pixels of subsets whose descriptor
  // has DG_DESC_EVOLVE set: 0 inactive (excluded), 1 active, 2 turned on
  // with the reference intensity in pix_f; evo_nact the subsets' counts of
  // pixels with state != 0
  uint8_t* pix_flag;
  float* pix_f;
  int32_t* evo_nact;
};

// ---------------------------------------------------------------------------
// Warp reductions
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ int warp_sum_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ int warp_min_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(FULL, v, o));
  return v;
}
__device__ __forceinline__ int warp_max_i(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(FULL, v, o));
  return v;
}

// ---------------------------------------------------------------------------
// FP64 tensor-core outer-product accumulation.
// mma.sync.m8n8k4 f64 (row.col): lane l holds A[l>>2][l&3], B[l&3][l>>2],
// and C/D[l>>2][2*(l&3) + {0,1}].  With A = V^T and B = V for four pixel
// vectors V (4 x 8), C accumulates sum_k v_k v_k^T.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile(
      "mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(c0), "+d"(c1)
      : "d"(a), "d"(b));
}

// ---------------------------------------------------------------------------
// Keys fourth-order kernel (DICe_Image.cpp:114-122), the published Keys
// (1981) 6-point cubic convolution kernel:
//   |s| < 1 :  4/3|s|^3 - 7/3|s|^2 + 1
//   |s| < 2 : -7/12|s|^3 + 3|s|^2 - 59/12|s| + 5/2
//   |s| < 3 :  1/12|s|^3 - 2/3|s|^2 + 7/4|s| - 3/2
// Two evaluations.  The *_ref ones are the reference's arithmetic: the
// kernel's coefficients as the 14-decimal literals it writes, products and
// sums in double, left to right, each rounded on its own, the result rounded
// to float.  The correlation path uses them, so that every interpolated value
// is the reference's bit for bit.  The FP32 Horner forms below them serve the
// adjoint, whose derivative pieces they match.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float keys_f0_ref(double s) {
  const double a = __dmul_rn(__dmul_rn(__dmul_rn(1.33333333333333, s), s), s);
  const double b = __dmul_rn(__dmul_rn(2.33333333333333, s), s);
  return __double2float_rn(__dadd_rn(__dsub_rn(a, b), 1.0));
}
__device__ __forceinline__ float keys_f1_ref(double s) {
  const double a = __dmul_rn(__dmul_rn(__dmul_rn(-0.58333333333333, s), s), s);
  const double b = __dmul_rn(__dmul_rn(3.0, s), s);
  const double c = __dmul_rn(4.91666666666666, s);
  return __double2float_rn(__dadd_rn(__dsub_rn(__dadd_rn(a, b), c), 2.5));
}
__device__ __forceinline__ float keys_f2_ref(double s) {
  const double a = __dmul_rn(__dmul_rn(__dmul_rn(0.08333333333333, s), s), s);
  const double b = __dmul_rn(__dmul_rn(0.66666666666666, s), s);
  const double c = __dmul_rn(1.75, s);
  return __double2float_rn(__dsub_rn(__dadd_rn(__dsub_rn(a, b), c), 1.5));
}
// The six weights of one axis at fractional offset d = x - (int)x, in the
// reference's argument order (DICe_Image.cpp:858-863), where each argument
// (d + 2.0 and so on) is rounded to float before the kernel sees it.
// Interior form: for x >= 2 the float spacing of x is at least 2^-22, so d
// and every k +- d (k = 0..3) is a multiple of 2^-22 in [0, 3]: exact in
// float, and the arguments can be formed in double from one conversion.
__device__ __forceinline__ void keys_weights_ref_interior(float d, float w[6]) {
  const double dd = (double)d;
  w[0] = keys_f2_ref(__dadd_rn(dd, 2.0));
  w[1] = keys_f1_ref(__dadd_rn(dd, 1.0));
  w[2] = keys_f0_ref(dd);
  w[3] = keys_f0_ref(__dsub_rn(1.0, dd));
  w[4] = keys_f1_ref(__dsub_rn(2.0, dd));
  w[5] = keys_f2_ref(__dsub_rn(3.0, dd));
}
// Any d >= 0: the arguments rounded to float first.  d + k and k - d are
// exact in double, so the float sum is the reference's (float)(d + k.0).
__device__ __forceinline__ void keys_weights_ref_general(float d, float w[6]) {
  w[0] = keys_f2_ref((double)__fadd_rn(d, 2.0f));
  w[1] = keys_f1_ref((double)__fadd_rn(d, 1.0f));
  w[2] = keys_f0_ref((double)d);
  w[3] = keys_f0_ref((double)__fsub_rn(1.0f, d));
  w[4] = keys_f1_ref((double)__fsub_rn(2.0f, d));
  w[5] = keys_f2_ref((double)__fsub_rn(3.0f, d));
}

__device__ __forceinline__ float keys0(float s) {
  return fmaf(fmaf(4.0f / 3.0f, s, -7.0f / 3.0f), s * s, 1.0f);
}
__device__ __forceinline__ float keys1(float s) {
  return fmaf(fmaf(fmaf(-7.0f / 12.0f, s, 3.0f), s, -59.0f / 12.0f), s, 2.5f);
}
__device__ __forceinline__ float keys2(float s) {
  return fmaf(fmaf(fmaf(1.0f / 12.0f, s, -2.0f / 3.0f), s, 1.75f), s, -1.5f);
}
__device__ __forceinline__ void keys_weights(float t, float w[6]) {
  w[0] = keys2(t + 2.0f);
  w[1] = keys1(t + 1.0f);
  w[2] = keys0(t);
  w[3] = keys0(1.0f - t);
  w[4] = keys1(2.0f - t);
  w[5] = keys2(3.0f - t);
}

// ---------------------------------------------------------------------------
// Reference-order interpolation (Image_::interpolate_*_all) at a point whose
// taps all lie inside the image (the subset border test keeps every active
// pixel at least 3.5 px from the edge, DICe_Subset.cpp:408).
// ---------------------------------------------------------------------------
// Keys-4 (DICe_Image.cpp:834-883): cc = wy[m] * wx[n] in float, then each
// channel += cc * tap, m outer, n inner.  With gradients the taps come from
// the interleaved (I, Gx, Gy, 0) image, one 16-byte load per tap.
template <bool GRAD>
__device__ __forceinline__ void keys_ref_interior(const DevImage& im, float x, float y, float& iv, float& gxv,
                                                  float& gyv) {
  const int ix = (int)x, iy = (int)y;
  float wx[6], wy[6];
  keys_weights_ref_interior(__fsub_rn(x, (float)ix), wx);
  keys_weights_ref_interior(__fsub_rn(y, (float)iy), wy);
  float a = 0.0f, b = 0.0f, c = 0.0f;
  if (GRAD) {
    const float4* q = im.p4 + (size_t)(iy - 2) * im.w + (ix - 2);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
#pragma unroll
      for (int n = 0; n < 6; ++n) {
        const float4 t = __ldg(q + n);
        const float cc = __fmul_rn(wy[m], wx[n]);
        a = __fadd_rn(a, __fmul_rn(cc, t.x));
        b = __fadd_rn(b, __fmul_rn(cc, t.y));
        c = __fadd_rn(c, __fmul_rn(cc, t.z));
      }
      q += im.w;
    }
  } else {
    const float* q = im.I + (size_t)(iy - 2) * im.w + (ix - 2);
#pragma unroll
    for (int m = 0; m < 6; ++m) {
#pragma unroll
      for (int n = 0; n < 6; ++n) a = __fadd_rn(a, __fmul_rn(__fmul_rn(wy[m], wx[n]), __ldg(q + n)));
      q += im.w;
    }
  }
  iv = a;
  gxv = b;
  gyv = c;
}

// Bilinear (DICe_Image.cpp:394-425): value = I11 (x2-x)(y2-y) + I21 (x-x1)(y2-y)
// + I22 (x-x1)(y-y1) + I12 (x2-x)(y-y1), each product left to right.
__device__ __forceinline__ float bilinear_ref(const float* __restrict__ a, int w, int x1, int y1, float fx2,
                                              float fx1, float fy2, float fy1) {
  const float* r1 = a + (size_t)y1 * w + x1;
  const float* r2 = r1 + w;
  float v = __fmul_rn(__fmul_rn(__ldg(r1), fx2), fy2);
  v = __fadd_rn(v, __fmul_rn(__fmul_rn(__ldg(r1 + 1), fx1), fy2));
  v = __fadd_rn(v, __fmul_rn(__fmul_rn(__ldg(r2 + 1), fx1), fy1));
  v = __fadd_rn(v, __fmul_rn(__fmul_rn(__ldg(r2), fx2), fy1));
  return v;
}

// Bicubic (DICe_Image.cpp:493-636).  The reference writes the Catmull-Rom
// (a = -1/2) bicubic as its expanded polynomial in x and y: the coefficient
// of x^a y^b is sum_{n,m} c_a[n] c_b[m] f(n, m) over the 4 x 4 taps, with the
// kernel's power-coefficient vectors
//   c_0 = (0, 1, 0, 0), c_1 = (-1/2, 0, 1/2, 0),
//   c_2 = (1, -5/2, 2, -1/2), c_3 = (-1/2, 3/2, -3/2, 1/2)
// (tap offsets -1, 0, 1, 2).  Each coefficient is summed over its nonzero
// terms, x tap outer and y tap inner, and the value is
//   f00 + C01 y + C02 y^2 + C03 y^3 + sum_{a=1..3} (Ca0 + Ca1 y + Ca2 y^2 + Ca3 y^3) x^a,
// every product and sum in float, left to right: the reference's order.
__device__ __forceinline__ float cr_coef(int a, int n) {
  // c_a[n] for a, n in 0..3 (compile-time after unrolling)
  return a == 0 ? (n == 1 ? 1.0f : 0.0f)
       : a == 1 ? (n == 0 ? -0.5f : n == 2 ? 0.5f : 0.0f)
       : a == 2 ? (n == 0 ? 1.0f : n == 1 ? -2.5f : n == 2 ? 2.0f : -0.5f)
                : (n == 0 ? -0.5f : n == 1 ? 1.5f : n == 2 ? -1.5f : 0.5f);
}
// f[n][m]: tap at x offset n - 1, y offset m - 1
__device__ __forceinline__ float bicubic_group(const float f[4][4], int a, int b) {
  float s = 0.0f;
  bool first = true;
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const float cf = cr_coef(a, n) * cr_coef(b, m);   // exact: products of the coefficients above
      if (cf == 0.0f) continue;
      const float t = __fmul_rn(cf, f[n][m]);
      s = first ? t : __fadd_rn(s, t);
      first = false;
    }
  return s;
}
__device__ __forceinline__ float bicubic_eval(const float f[4][4], float x, float y) {
  const float x2 = __fmul_rn(x, x), x3 = __fmul_rn(x2, x);
  const float y2 = __fmul_rn(y, y), y3 = __fmul_rn(y2, y);
  float v = f[1][1];
  v = __fadd_rn(v, __fmul_rn(bicubic_group(f, 0, 1), y));
  v = __fadd_rn(v, __fmul_rn(bicubic_group(f, 0, 2), y2));
  v = __fadd_rn(v, __fmul_rn(bicubic_group(f, 0, 3), y3));
  const float xp[4] = {1.0f, x, x2, x3};
#pragma unroll
  for (int a = 1; a < 4; ++a) {
    float g = bicubic_group(f, a, 0);
    g = __fadd_rn(g, __fmul_rn(bicubic_group(f, a, 1), y));
    g = __fadd_rn(g, __fmul_rn(bicubic_group(f, a, 2), y2));
    g = __fadd_rn(g, __fmul_rn(bicubic_group(f, a, 3), y3));
    v = __fadd_rn(v, __fmul_rn(g, xp[a]));
  }
  return v;
}
template <bool GRAD>
__device__ __forceinline__ void bicubic_ref_interior(const DevImage& im, float lx, float ly, float& iv, float& gxv,
                                                     float& gyv) {
  const int x0 = (int)lx, y0 = (int)ly;
  const float x = __fsub_rn(lx, (float)x0), y = __fsub_rn(ly, (float)y0);
  float f[4][4];
  const size_t base = (size_t)(y0 - 1) * im.w + (x0 - 1);
#pragma unroll
  for (int n = 0; n < 4; ++n)
#pragma unroll
    for (int m = 0; m < 4; ++m) f[n][m] = __ldg(im.I + base + (size_t)m * im.w + n);
  iv = bicubic_eval(f, x, y);
  if (GRAD) {
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int m = 0; m < 4; ++m) f[n][m] = __ldg(im.gx + base + (size_t)m * im.w + n);
    gxv = bicubic_eval(f, x, y);
#pragma unroll
    for (int n = 0; n < 4; ++n)
#pragma unroll
      for (int m = 0; m < 4; ++m) f[n][m] = __ldg(im.gy + base + (size_t)m * im.w + n);
    gyv = bicubic_eval(f, x, y);
  }
}

// Interpolation of the correlation path in the reference's arithmetic.
template <int INTERP, bool GRAD>
__device__ __forceinline__ void interp_ref(const DevImage& im, float x, float y, float& iv, float& gxv,
                                           float& gyv) {
  if (INTERP == DICEGPU_KEYS_FOURTH) {
    keys_ref_interior<GRAD>(im, x, y, iv, gxv, gyv);
  } else if (INTERP == DICEGPU_BICUBIC) {
    bicubic_ref_interior<GRAD>(im, x, y, iv, gxv, gyv);
  } else {
    const int x1 = (int)x, y1 = (int)y;
    const float fx2 = __fsub_rn((float)(x1 + 1), x), fx1 = __fsub_rn(x, (float)x1);
    const float fy2 = __fsub_rn((float)(y1 + 1), y), fy1 = __fsub_rn(y, (float)y1);
    iv = bilinear_ref(im.I, im.w, x1, y1, fx2, fx1, fy2, fy1);
    if (GRAD) {
      gxv = bilinear_ref(im.gx, im.w, x1, y1, fx2, fx1, fy2, fy1);
      gyv = bilinear_ref(im.gy, im.w, x1, y1, fx2, fx1, fy2, fy1);
    }
  }
}

// FP32 separable evaluation (fused multiply-adds, a row sum per row), the
// adjoint's forward map.
template <int R, bool GRAD>
__device__ __forceinline__ void conv_taps(const DevImage& im, int x0, int y0, const float* wx,
                                          const float* wy, float& iv, float& gxv, float& gyv) {
  const int w = im.w;
  float a = 0.0f, b = 0.0f, c = 0.0f;
  if (GRAD) {
    const float4* q = im.p4 + (size_t)y0 * w + x0;
#pragma unroll
    for (int m = 0; m < R; ++m) {
      float ra = 0.0f, rb = 0.0f, rc = 0.0f;
#pragma unroll
      for (int n = 0; n < R; ++n) {
        const float4 t = __ldg(q + n);
        ra = fmaf(wx[n], t.x, ra);
        rb = fmaf(wx[n], t.y, rb);
        rc = fmaf(wx[n], t.z, rc);
      }
      a = fmaf(wy[m], ra, a);
      b = fmaf(wy[m], rb, b);
      c = fmaf(wy[m], rc, c);
      q += w;
    }
    gxv = b;
    gyv = c;
  } else {
    const float* q = im.I + (size_t)y0 * w + x0;
#pragma unroll
    for (int m = 0; m < R; ++m) {
      float ra = 0.0f;
#pragma unroll
      for (int n = 0; n < R; ++n) ra = fmaf(wx[n], __ldg(q + n), ra);
      a = fmaf(wy[m], ra, a);
      q += w;
    }
  }
  iv = a;
}

// Keys-4 in the separable FP32 form (the adjoint's forward map).
template <bool GRAD>
__device__ __forceinline__ void keys_fast_interior(const DevImage& im, float x, float y, float& iv, float& gxv,
                                                   float& gyv) {
  const int ix = (int)x, iy = (int)y;
  float wx[6], wy[6];
  keys_weights(x - (float)ix, wx);
  keys_weights(y - (float)iy, wy);
  conv_taps<6, GRAD>(im, ix - 2, iy - 2, wx, wy, iv, gxv, gyv);
}

// Float cosine, sine and arc cosine as the double functions rounded to float:
// correctly rounded but for arguments within about 2^-28 ulp of a rounding
// boundary, like the C library's float versions the reference calls
// (std::cos(float) and so on), so both sides agree on the float values.
__device__ __forceinline__ float cos_f(float t) { return (float)cos((double)t); }
__device__ __forceinline__ float sin_f(float t) { return (float)sin((double)t); }
__device__ __forceinline__ float acos_f(float t) { return (float)acos((double)t); }

// ---------------------------------------------------------------------------
// Shape functions.
// ---------------------------------------------------------------------------
// Per-pass constants of the current parameters (uniform across the warp).
struct MapConst {
  float s[12];   // slots
  float cost, sint;
  float rcos, rsin;  // rotation of reference gradients (use_ref_grads)
};

// Affine_Shape_Function::map (DICe_LocalShapeFunction.cpp:220-248).  The
// stretch terms are formed in double exactly as the reference's (1.0+dudx)
// literal makes them; the rest is FP32 without contraction so the mapped
// coordinate (and hence pixel rounding / deactivation) matches bit for bit.
__device__ __forceinline__ void affine_D(const MapConst& k, float dx, float dy, float& Dx,
                                         float& Dy) {
  Dx = (float)__dadd_rn(__dmul_rn(1.0 + (double)k.s[3], (double)dx), (double)__fmul_rn(k.s[5], dy));
  Dy = (float)__dadd_rn(__dmul_rn(1.0 + (double)k.s[4], (double)dy), (double)__fmul_rn(k.s[5], dx));
}

// Map of a pixel offset (dx, dy) = (x - cx, y - cy); for affine maps the
// stretched offsets (Dx, Dy) are returned too (the residuals reuse them).
template <int SHAPE>
__device__ __forceinline__ void map_offset(const MapConst& k, float dx, float dy, float cx, float cy,
                                           float& ox, float& oy, float& Dx, float& Dy) {
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    // Quadratic_Shape_Function::map (:509-520), left-to-right FP32 sums
    float a = __fmul_rn(k.s[0], dx);
    a = __fadd_rn(a, __fmul_rn(k.s[1], dy));
    a = __fadd_rn(a, __fmul_rn(__fmul_rn(k.s[2], dx), dy));
    a = __fadd_rn(a, __fmul_rn(__fmul_rn(k.s[3], dx), dx));
    a = __fadd_rn(a, __fmul_rn(__fmul_rn(k.s[4], dy), dy));
    a = __fadd_rn(a, k.s[5]);
    ox = __fadd_rn(a, cx);
    float b = __fmul_rn(k.s[6], dx);
    b = __fadd_rn(b, __fmul_rn(k.s[7], dy));
    b = __fadd_rn(b, __fmul_rn(__fmul_rn(k.s[8], dx), dy));
    b = __fadd_rn(b, __fmul_rn(__fmul_rn(k.s[9], dx), dx));
    b = __fadd_rn(b, __fmul_rn(__fmul_rn(k.s[10], dy), dy));
    b = __fadd_rn(b, k.s[11]);
    oy = __fadd_rn(b, cy);
    Dx = dx;
    Dy = dy;
  } else {
    affine_D(k, dx, dy, Dx, Dy);
    ox = __fadd_rn(__fadd_rn(__fsub_rn(__fmul_rn(k.cost, Dx), __fmul_rn(k.sint, Dy)), k.s[0]), cx);
    oy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(k.sint, Dx), __fmul_rn(k.cost, Dy)), k.s[1]), cy);
  }
}

// Residual vector dG/dp in slot order (affine :350-396, quadratic :580-614)
// from the pixel offset and the stretched offset of map_offset.
template <int SHAPE>
__device__ __forceinline__ void residuals_D(const MapConst& k, float dx, float dy, float Dx, float Dy,
                                            float gx, float gy, bool use_ref_grads, float* r) {
  float Gx = gx, Gy = gy;
  if (use_ref_grads) {
    Gx = k.rcos * gx - k.rsin * gy;
    Gy = k.rsin * gx + k.rcos * gy;
  }
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    // Gx*dx*dy is (Gx*dx)*dy, left to right, as the reference writes it
    r[0] = Gx * dx; r[1] = Gx * dy; r[2] = Gx * dx * dy; r[3] = Gx * dx * dx; r[4] = Gx * dy * dy; r[5] = Gx;
    r[6] = Gy * dx; r[7] = Gy * dy; r[8] = Gy * dx * dy; r[9] = Gy * dx * dx; r[10] = Gy * dy * dy; r[11] = Gy;
  } else {
    const float c = k.cost, s = k.sint;
    r[0] = Gx;
    r[1] = Gy;
    r[2] = Gx * (-s * Dx - c * Dy) + Gy * (c * Dx - s * Dy);
    r[3] = Gx * dx * c + Gy * dx * s;
    r[4] = -Gx * dy * s + Gy * dy * c;
    r[5] = Gx * (c * dy - s * dx) + Gy * (s * dy + c * dx);
  }
}

template <int SHAPE>
__device__ __forceinline__ void map_point(const MapConst& k, float x, float y, float cx, float cy,
                                          float& ox, float& oy) {
  const float dx = __fsub_rn(x, cx), dy = __fsub_rn(y, cy);
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    // Quadratic_Shape_Function::map (:509-520), left-to-right FP32 sums
    const float dxdy = __fmul_rn(dx, dy), dx2 = __fmul_rn(dx, dx), dy2 = __fmul_rn(dy, dy);
    float a = __fmul_rn(k.s[0], dx);
    a = __fadd_rn(a, __fmul_rn(k.s[1], dy));
    a = __fadd_rn(a, __fmul_rn(__fmul_rn(k.s[2], dx), dy));
    a = __fadd_rn(a, __fmul_rn(__fmul_rn(k.s[3], dx), dx));
    a = __fadd_rn(a, __fmul_rn(__fmul_rn(k.s[4], dy), dy));
    a = __fadd_rn(a, k.s[5]);
    ox = __fadd_rn(a, cx);
    float b = __fmul_rn(k.s[6], dx);
    b = __fadd_rn(b, __fmul_rn(k.s[7], dy));
    b = __fadd_rn(b, __fmul_rn(__fmul_rn(k.s[8], dx), dy));
    b = __fadd_rn(b, __fmul_rn(__fmul_rn(k.s[9], dx), dx));
    b = __fadd_rn(b, __fmul_rn(__fmul_rn(k.s[10], dy), dy));
    b = __fadd_rn(b, k.s[11]);
    oy = __fadd_rn(b, cy);
    (void)dxdy; (void)dx2; (void)dy2;
  } else {
    float Dx, Dy;
    affine_D(k, dx, dy, Dx, Dy);
    ox = __fadd_rn(__fadd_rn(__fsub_rn(__fmul_rn(k.cost, Dx), __fmul_rn(k.sint, Dy)), k.s[0]), cx);
    oy = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(k.sint, Dx), __fmul_rn(k.cost, Dy)), k.s[1]), cy);
  }
}

// Residual vector dG/dp in slot order (affine :350-396, quadratic :580-614).
template <int SHAPE>
__device__ __forceinline__ void residuals(const MapConst& k, float x, float y, float cx, float cy,
                                          float gx, float gy, bool use_ref_grads, float* r) {
  const float dx = x - cx, dy = y - cy;
  float Gx = gx, Gy = gy;
  if (use_ref_grads) {
    Gx = k.rcos * gx - k.rsin * gy;
    Gy = k.rsin * gx + k.rcos * gy;
  }
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    // Gx*dx*dy is (Gx*dx)*dy, left to right, as the reference writes it
    r[0] = Gx * dx; r[1] = Gx * dy; r[2] = Gx * dx * dy; r[3] = Gx * dx * dx; r[4] = Gx * dy * dy; r[5] = Gx;
    r[6] = Gy * dx; r[7] = Gy * dy; r[8] = Gy * dx * dy; r[9] = Gy * dx * dx; r[10] = Gy * dy * dy; r[11] = Gy;
  } else {
    float Dx, Dy;
    affine_D(k, dx, dy, Dx, Dy);
    const float c = k.cost, s = k.sint;
    r[0] = Gx;
    r[1] = Gy;
    r[2] = Gx * (-s * Dx - c * Dy) + Gy * (c * Dx - s * Dy);
    r[3] = Gx * dx * c + Gy * dx * s;
    r[4] = -Gx * dy * s + Gy * dy * c;
    r[5] = Gx * (c * dy - s * dx) + Gy * (s * dy + c * dx);
  }
}

// Quadratic_Shape_Function::map_to_u_v_theta (:552-578); affine reads slots.
template <int SHAPE>
__device__ __forceinline__ void map_to_u_v_theta(const MapConst& k, float cx, float cy, float& u,
                                                 float& v, float& t) {
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    float cxp, cyp, rxp, ryp;
    map_point<SHAPE>(k, cx, cy, cx, cy, cxp, cyp);
    u = cxp - cx;
    v = cyp - cy;
    map_point<SHAPE>(k, (float)((double)cx + 5.0), cy, cx, cy, rxp, ryp);
    const float ax = rxp - cxp, ay = ryp - cyp;
    const float mag_a = sqrtf(ax * ax + ay * ay);
    const float adb = (ax * 5.0f + ay * 0.0f) / (mag_a * 5.0f);
    t = ay < 0.0f ? (float)(6.28318530717958647692 - (double)acos_f(adb)) : acos_f(adb);
  } else {
    u = k.s[0];
    v = k.s[1];
    t = k.s[2];
  }
}

template <int SHAPE>
__device__ __forceinline__ void make_mapconst(const float* slots, bool use_ref_grads, float cx,
                                              float cy, MapConst& k) {
#pragma unroll
  for (int i = 0; i < 12; ++i) k.s[i] = slots[i];
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    k.cost = 1.0f; k.sint = 0.0f;
    k.rcos = 1.0f; k.rsin = 0.0f;
    if (use_ref_grads) {
      float u, v, t;
      map_to_u_v_theta<SHAPE>(k, cx, cy, u, v, t);
      k.rcos = cos_f(t);
      k.rsin = sin_f(t);
    }
  } else {
    k.cost = cos_f(slots[2]);
    k.sint = sin_f(slots[2]);
    k.rcos = k.cost;
    k.rsin = k.sint;
  }
}

// angle_2d (DICe_Shape.cpp:87-102) in the reference's precision, with the
// float atan2 correctly rounded (the double atan2 rounded to float) so that
// pixels lying exactly on a polygon edge, whose edge term is +-pi, are
// decided the same way as on the host.
__device__ __forceinline__ float polygon_angle(float x1, float y1, float x2, float y2) {
  const float t1 = (float)atan2((double)y1, (double)x1), t2 = (float)atan2((double)y2, (double)x2);
  float d = __fsub_rn(t2, t1);
  for (int k = 0; k < 4 && (double)d > 3.14159265358979323846; ++k) d = (float)((double)d - 6.28318530717958647692);
  for (int k = 0; k < 4 && (double)d < -3.14159265358979323846; ++k) d = (float)((double)d + 6.28318530717958647692);
  return d;
}

// winding-angle test over a closed vertex loop (vertex nv is vertex 0)
__device__ __forceinline__ bool polygon_has(const int32_t* ax, const int32_t* ay, int nv, int x, int y) {
  float angle = 0.0f;
  for (int i = 0; i < nv; ++i) {
    const int j = (i + 1 == nv) ? 0 : i + 1;
    angle = __fadd_rn(angle, polygon_angle((float)(ax[i] - x), (float)(ay[i] - y), (float)(ax[j] - x),
                                          (float)(ay[j] - y)));
  }
  return (double)fabsf(angle) >= 3.14159265358979323846;
}

// Pixel rounding of Subset::initialize (DICe_Subset.cpp:405-406).
// The reference adds 0.5 in double; in float m + 0.5f is exact for
// |m| < 2^22 except where the sum crosses a power of two, and there the
// rounding cannot cross an integer, so the truncations agree.
__device__ __forceinline__ int round_pixel(float m) {
  const int a = (int)m;
  const int b = (int)(m + 0.5f);
  return b == a ? a : a + 1;
}

}  // namespace dg
