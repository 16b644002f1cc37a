// dg_device.cuh -- device building blocks of the subset-correlation path.
//
// Warp-per-subset design: one warp owns one subset at a time.  Lanes take
// 32 subset pixels per step; warp-wide results come from shuffles and from
// FP64 tensor-core accumulation (mma.sync m8n8k4 f64), so no block-level
// synchronisation exists anywhere on the hot path.
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
  const uint8_t* __restrict__ force_simplex;
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
// in Horner form, FP32.
// ---------------------------------------------------------------------------
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
// Catmull-Rom (a = -1/2) weights: the separable form of the bicubic
// polynomial of Image_::interpolate_bicubic_all (DICe_Image.cpp:493-636).
__device__ __forceinline__ void cubic_weights(float t, float w[4]) {
  const float t2 = t * t, t3 = t2 * t;
  w[0] = 0.5f * (-t3 + 2.0f * t2 - t);
  w[1] = 0.5f * (3.0f * t3 - 5.0f * t2 + 2.0f);
  w[2] = 0.5f * (-3.0f * t3 + 4.0f * t2 + t);
  w[3] = 0.5f * (t3 - t2);
}

// Interpolation at an interior point (the subset border test keeps every
// active pixel at least 3.5 px from the image edge, so no tap leaves the
// image: DICe_Subset.cpp:408).  Separable evaluation: a 6-tap (4-tap) row sum
// per row, then the column sum.  With gradients the taps come from the
// interleaved (I, Gx, Gy, 0) image, one 16-byte load per tap.
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

template <int INTERP, bool GRAD>
__device__ __forceinline__ void interp_interior(const DevImage& im, float x, float y, float& iv,
                                                float& gxv, float& gyv) {
  const int ix = (int)x, iy = (int)y;
  if (INTERP == DICEGPU_KEYS_FOURTH) {
    float wx[6], wy[6];
    keys_weights(x - (float)ix, wx);
    keys_weights(y - (float)iy, wy);
    conv_taps<6, GRAD>(im, ix - 2, iy - 2, wx, wy, iv, gxv, gyv);
  } else if (INTERP == DICEGPU_BICUBIC) {
    float wx[4], wy[4];
    cubic_weights(x - (float)ix, wx);
    cubic_weights(y - (float)iy, wy);
    conv_taps<4, GRAD>(im, ix - 1, iy - 1, wx, wy, iv, gxv, gyv);
  } else {
    // Image_::interpolate_bilinear_all (DICe_Image.cpp:394-425), interior form
    const float fx1 = (float)(ix + 1) - x, fx0 = x - (float)ix;
    const float fy1 = (float)(iy + 1) - y, fy0 = y - (float)iy;
    const float wx[2] = {fx1, fx0}, wy[2] = {fy1, fy0};
    conv_taps<2, GRAD>(im, ix, iy, wx, wy, iv, gxv, gyv);
  }
}

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
    const float dxdy = dx * dy, dx2 = dx * dx, dy2 = dy * dy;
    r[0] = Gx * dx; r[1] = Gx * dy; r[2] = Gx * dxdy; r[3] = Gx * dx2; r[4] = Gx * dy2; r[5] = Gx;
    r[6] = Gy * dx; r[7] = Gy * dy; r[8] = Gy * dxdy; r[9] = Gy * dx2; r[10] = Gy * dy2; r[11] = Gy;
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
    const float dxdy = dx * dy, dx2 = dx * dx, dy2 = dy * dy;
    r[0] = Gx * dx; r[1] = Gx * dy; r[2] = Gx * dxdy; r[3] = Gx * dx2; r[4] = Gx * dy2; r[5] = Gx;
    r[6] = Gy * dx; r[7] = Gy * dy; r[8] = Gy * dxdy; r[9] = Gy * dx2; r[10] = Gy * dy2; r[11] = Gy;
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
    t = ay < 0.0f ? (float)(6.28318530717958647692 - (double)acosf(adb)) : acosf(adb);
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
      k.rcos = cosf(t);
      k.rsin = sinf(t);
    }
  } else {
    k.cost = cosf(slots[2]);
    k.sint = sinf(slots[2]);
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
