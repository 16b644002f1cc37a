// dice_oracle.cpp -- CPU oracle for the DICe local subset-correlation path.
//
// TEST INFRASTRUCTURE ONLY: the checker for tests/, smoke() and the CPU
// baseline leg of bench.py.  Never linked into or called by libdicegpu.so.
//
// It restates, function by function, the reference's CPU path with the
// reference's precision contract: scalar_t = float for warp, interpolation,
// residuals and products; double for the Gauss-Newton Hessian / RHS and the
// LU factorisation (DICe.h:96-118, DICe_Objective.cpp:448-449).  It is built
// with -ffp-contract=off so that no fused multiply-add changes a rounding the
// reference's x86-64 build would not change.  Citations are paths inside the
// DICe project.
//
// Deliberate reference behaviours kept here (each also kept by the GPU path):
//  * pixel rounding (int)(x+0.5)==(int)x ? (int)x : (int)x+1 and the 4-pixel
//    border deactivation (DICe_Subset.cpp:405-411);
//  * GN runs solve_it = 0..max inclusive and reports the last index
//    (DICe_Objective.cpp:494-495, 653);
//  * the affine convergence test reads only u, v, theta
//    (DICe_LocalShapeFunction.cpp:433-459);
//  * the singular-Hessian test uses only the 2x2 displacement block
//    (DICe_Objective.cpp:558-579) and the GETRF info code is ignored;
//  * on success STATUS_FLAG is the initializer's status (DICe_Schema.cpp:2351);
//  * SIGMA = -1 after a failed frame makes the next initial guess fail with
//    INITIALIZE_FAILED (DICe_Initializer.cpp:415-435);
//  * noise_std_dev's bounding-box quirks (DICe_Subset.cpp:664-684);
//  * the simplex leaves the shape function at the last point it evaluated
//    (the variables alias the parameters, DICe_LocalShapeFunction.h:259-261).
#include "dice_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <thread>
#include <set>
#include <vector>

namespace oracle {

static const double kPi = 3.14159265358979323846;
static const double kTwoPi = 6.28318530717958647692;

// ---------------------------------------------------------------------------
// Image (DICe_Image.cpp)
// ---------------------------------------------------------------------------
struct Image {
  int w = 0, h = 0;
  const float* I = nullptr;
  const float* gx = nullptr;
  const float* gy = nullptr;
  bool has_gradients = false;
  // linear-index read: the reference indexes intensities_[y*w+x] without a
  // bounds check; inside the array we read the same element, outside (only
  // reachable through paths the subset border test excludes) we read 0.
  inline float at(const float* a, long idx) const {
    return (idx >= 0 && idx < (long)w * h) ? a[idx] : 0.0f;
  }
};

// Keys fourth-order cubic convolution kernel pieces (DICe_Image.cpp:114-122).
// The published Keys (1981) 6-point kernel: for s in [0,1): 4/3 s^3 - 7/3 s^2 + 1;
// [1,2): -7/12 s^3 + 3 s^2 - 59/12 s + 5/2; [2,3): 1/12 s^3 - 2/3 s^2 + 7/4 s - 3/2,
// with the coefficients written as the 14-decimal literals the reference uses,
// evaluated in double left to right and rounded to float, as its double
// literals make it.
static inline float keys_f0(float s) {
  return (float)(1.33333333333333 * s * s * s - 2.33333333333333 * s * s + 1.0);
}
static inline float keys_f1(float s) {
  return (float)(-0.58333333333333 * s * s * s + 3.0 * s * s - 4.91666666666666 * s + 2.5);
}
static inline float keys_f2(float s) {
  return (float)(0.08333333333333 * s * s * s - 0.66666666666666 * s * s + 1.75 * s - 1.5);
}

// Image_::interpolate_bilinear (DICe_Image.cpp:432-445) on one channel.
static float bilinear(const Image& im, const float* a, float lx, float ly) {
  if (lx < 0.0 || lx >= im.w - 1.5 || ly < 0.0 || ly >= im.h - 1.5) return 0.0f;
  const int x1 = (int)lx, x2 = x1 + 1, y1 = (int)ly, y2 = y1 + 1;
  const int w = im.w;
  return a[y1 * w + x1] * (x2 - lx) * (y2 - ly) + a[y1 * w + x2] * (lx - x1) * (y2 - ly) +
         a[y2 * w + x2] * (lx - x1) * (ly - y1) + a[y2 * w + x1] * (x2 - lx) * (ly - y1);
}

// Image_::interpolate_bilinear_all (DICe_Image.cpp:394-425).
static void interp_bilinear_all(const Image& im, float& iv, float& gxv, float& gyv, bool grad,
                                float lx, float ly) {
  iv = bilinear(im, im.I, lx, ly);
  if (grad) {
    gxv = bilinear(im, im.gx, lx, ly);
    gyv = bilinear(im, im.gy, lx, ly);
  }
}

// Image_::interpolate_bicubic_all (DICe_Image.cpp:493-636).  The reference
// writes the Catmull-Rom (a = -1/2) bicubic as its polynomial expanded in x
// and y: the coefficient of x^a y^b is sum_{n,m} c_a[n] c_b[m] f(n, m) over
// the 4 x 4 taps (offsets -1..2), with the kernel's power-coefficient vectors
//   c_0 = (0, 1, 0, 0), c_1 = (-1/2, 0, 1/2, 0),
//   c_2 = (1, -5/2, 2, -1/2), c_3 = (-1/2, 3/2, -3/2, 1/2).
// Each coefficient sums its nonzero terms with the x tap outer and the y
// tap inner, and the value is
//   f00 + C01 y + C02 y^2 + C03 y^3 + sum_{a=1..3} (Ca0 + Ca1 y + Ca2 y^2 + Ca3 y^3) x^a,
// every product and sum in float, left to right: the reference's expression
// order.  The coefficients' products are exact in float.
static const float kCR[4][4] = {{0.0f, 1.0f, 0.0f, 0.0f},
                                {-0.5f, 0.0f, 0.5f, 0.0f},
                                {1.0f, -2.5f, 2.0f, -0.5f},
                                {-0.5f, 1.5f, -1.5f, 0.5f}};
static float bicubic_group(const float f[4][4], int a, int b) {
  float s = 0.0f;
  bool first = true;
  for (int n = 0; n < 4; ++n)
    for (int m = 0; m < 4; ++m) {
      const float cf = kCR[a][n] * kCR[b][m];
      if (cf == 0.0f) continue;
      const float t = cf * f[n][m];
      s = first ? t : s + t;
      first = false;
    }
  return s;
}
static float bicubic_channel(const Image& im, const float* a, int x0, int y0, float x, float y) {
  float f[4][4];   // f[n][m]: tap at x offset n - 1, y offset m - 1
  for (int n = 0; n < 4; ++n)
    for (int m = 0; m < 4; ++m) f[n][m] = im.at(a, (long)(y0 - 1 + m) * im.w + (x0 - 1 + n));
  const float x2 = x * x, x3 = x2 * x, y2 = y * y, y3 = y2 * y;
  float v = f[1][1];
  v = v + bicubic_group(f, 0, 1) * y;
  v = v + bicubic_group(f, 0, 2) * y2;
  v = v + bicubic_group(f, 0, 3) * y3;
  const float xp[4] = {1.0f, x, x2, x3};
  for (int a = 1; a < 4; ++a) {
    float g = bicubic_group(f, a, 0);
    g = g + bicubic_group(f, a, 1) * y;
    g = g + bicubic_group(f, a, 2) * y2;
    g = g + bicubic_group(f, a, 3) * y3;
    v = v + g * xp[a];
  }
  return v;
}

// The reference computes a bilinear fallback near the border and then falls
// through to the bicubic expression, which overwrites it; we do the same.
static void interp_bicubic_all(const Image& im, float& iv, float& gxv, float& gyv, bool grad,
                               float lx, float ly) {
  const int x0 = (int)lx, y0 = (int)ly;
  const float x = lx - x0, y = ly - y0;
  iv = bicubic_channel(im, im.I, x0, y0, x, y);
  if (grad) {
    gxv = bicubic_channel(im, im.gx, x0, y0, x, y);
    gyv = bicubic_channel(im, im.gy, x0, y0, x, y);
  }
}

// Image_::interpolate_keys_fourth_all (DICe_Image.cpp:834-883): 6x6 taps,
// cc = wy[m]*wx[n] in float, accumulated m-outer / n-inner in float.  As in
// the reference the bilinear border value is overwritten by the Keys sum.
static void interp_keys_all(const Image& im, float& iv, float& gxv, float& gyv, bool grad,
                            float lx, float ly) {
  iv = 0.0f;
  if (grad) { gxv = 0.0f; gyv = 0.0f; }
  const int ix = (int)lx, iy = (int)ly;
  const float dx = lx - ix, dy = ly - iy;
  float cx[6], cy[6];
  cx[0] = keys_f2((float)(dx + 2.0));
  cx[1] = keys_f1((float)(dx + 1.0));
  cx[2] = keys_f0(dx);
  cx[3] = keys_f0((float)(1.0 - dx));
  cx[4] = keys_f1((float)(2.0 - dx));
  cx[5] = keys_f2((float)(3.0 - dx));
  cy[0] = keys_f2((float)(dy + 2.0));
  cy[1] = keys_f1((float)(dy + 1.0));
  cy[2] = keys_f0(dy);
  cy[3] = keys_f0((float)(1.0 - dy));
  cy[4] = keys_f1((float)(2.0 - dy));
  cy[5] = keys_f2((float)(3.0 - dy));
  for (int m = 0; m < 6; ++m) {
    for (int n = 0; n < 6; ++n) {
      const float cc = cy[m] * cx[n];
      const long idx = (long)(iy - 2 + m) * im.w + ix - 2 + n;
      iv += cc * im.at(im.I, idx);
      if (grad) {
        gxv += cc * im.at(im.gx, idx);
        gyv += cc * im.at(im.gy, idx);
      }
    }
  }
}

static void interpolate(const Image& im, int method, float& iv, float& gxv, float& gyv, bool grad,
                        float lx, float ly) {
  switch (method) {
    case DICEGPU_BILINEAR: interp_bilinear_all(im, iv, gxv, gyv, grad, lx, ly); break;
    case DICEGPU_BICUBIC: interp_bicubic_all(im, iv, gxv, gyv, grad, lx, ly); break;
    default: interp_keys_all(im, iv, gxv, gyv, grad, lx, ly); break;
  }
}

// Image_::compute_gradients_finite_difference (DICe_Image.cpp:1066-1093) with
// grad_c1 = 1/12, grad_c2 = -8/12 stored as float (DICe_Image.cpp:214-215),
// then optional 5x5 smoothing (smooth_gradients_convolution_5_point, :1034-1060).
static void compute_gradients(int w, int h, const float* I, int method, float* gx, float* gy) {
  const float c1 = (float)(1.0 / 12.0), c2 = (float)(-8.0 / 12.0);
  for (int y = 0; y < h; ++y) {
    for (int x = 0; x < w; ++x) {
      const long i = (long)y * w + x;
      if (x < 2) gx[i] = I[i + 1] - I[i];
      else if (x >= w - 2) gx[i] = I[i] - I[i - 1];
      else gx[i] = c1 * I[i - 2] + c2 * I[i - 1] - c2 * I[i + 1] - c1 * I[i + 2];
      if (y < 2) gy[i] = I[i + w] - I[i];
      else if (y >= h - 2) gy[i] = I[i] - I[i - w];
      else gy[i] = c1 * I[i - 2 * w] + c2 * I[i - w] - c2 * I[i + w] - c1 * I[i + 2 * w];
    }
  }
  if (method == DICEGPU_CONVOLUTION_5_POINT) {
    // binomial 5-tap smoothing, outer product of (1,4,6,4,1)/16
    static const float k[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
    std::vector<float> tx(gx, gx + (long)w * h), ty(gy, gy + (long)w * h);
    for (int y = 2; y < h - 2; ++y) {
      for (int x = 2; x < w - 2; ++x) {
        float vx = 0.0f, vy = 0.0f;
        for (int i = 0; i < 5; ++i)
          for (int j = 0; j < 5; ++j) {
            const float c = k[i] * k[j];
            const long idx = (long)(y + i - 2) * w + x + j - 2;
            vx += c * tx[idx];
            vy += c * ty[idx];
          }
        gx[(long)y * w + x] = vx;
        gy[(long)y * w + x] = vy;
      }
    }
  }
}

// Mask of Image_::gauss_filter (DICe_Image.cpp:54-112): the reference's
// tables are outer products of these 1-D weights, each printed to 9
// significant digits, stored as float.
static bool gauss_mask(int M, std::vector<float>& c) {
  static const double h5[] = {0.0014, 0.1574, 0.62825};
  static const double h7[] = {0.006, 0.0606, 0.2418, 0.3831};
  static const double h9[] = {0.0007, 0.0108, 0.0748, 0.2384, 0.3505};
  static const double h11[] = {0.0001, 0.0017, 0.0168, 0.087, 0.2328, 0.3231};
  static const double h13[] = {0.0001, 0.0012, 0.0085, 0.038, 0.1109, 0.2108, 0.2611};
  const double* hw = M == 5 ? h5 : M == 7 ? h7 : M == 9 ? h9 : M == 11 ? h11 : M == 13 ? h13 : nullptr;
  if (!hw) return false;
  c.assign((size_t)M * M, 0.0f);
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < M; ++j) {
      const double a = hw[i <= M / 2 ? i : M - 1 - i], b = hw[j <= M / 2 ? j : M - 1 - j];
      char buf[32];
      std::snprintf(buf, sizeof(buf), "%.8e", a * b);
      c[(size_t)i * M + j] = (float)std::strtod(buf, nullptr);
    }
  return true;
}

// Image_::gauss_filter (DICe_Image.cpp:1194-1230): interior pixels (at least
// M/2+1 from every edge) get the mask sum of the unfiltered copy, x offset
// outer and y offset inner, in float; the rest keep their value.
static bool gauss_filter(int w, int h, int M, const float* in, float* out) {
  std::vector<float> c;
  if (!gauss_mask(M, c) || w < M || h < M) return false;
  const int half = M / 2 + 1;
  std::vector<float> tmp(in, in + (long)w * h);
  for (int y = 0; y < h; ++y)
    for (int x = 0; x < w; ++x) {
      const long o = (long)y * w + x;
      if (x >= half && x < w - half && y >= half && y < h - half) {
        float v = 0.0f;
        for (int i = 0; i < M; ++i)
          for (int j = 0; j < M; ++j)
            v += c[(size_t)i * M + j] * tmp[(long)(y + j - half + 1) * w + x + i - half + 1];
        out[o] = v;
      } else {
        out[o] = tmp[o];
      }
    }
  return true;
}

// Float cosine, sine and arc cosine of the shape functions, taken correctly
// rounded: the double function rounded to float.  The reference calls the
// C library's float versions (std::cos(float) and so on; its affine map's
// unqualified cos(theta) may resolve to the double one), which are not
// correctly rounded for every argument and differ between library versions,
// so the reference's own rotated results depend on the libm it links; the
// correctly rounded value is the same on every platform and on the GPU.
static inline float cos_f(float t) { return (float)std::cos((double)t); }
static inline float sin_f(float t) { return (float)std::sin((double)t); }
static inline float acos_f(float t) { return (float)std::acos((double)t); }

// ---------------------------------------------------------------------------
// Local shape functions (DICe_LocalShapeFunction.cpp)
// ---------------------------------------------------------------------------
struct ShapeFn {
  int type = DICEGPU_AFFINE_SF;
  int N = 2;
  // affine parameter slots in spec_map_ insertion order (init, :170-218)
  int iu = 0, iv = 1, it = -1, iex = -1, iey = -1, ig = -1;
  float p[12];
  float deltas[12];

  void init(const dicegpu_params& P) {
    type = P.shape_function;
    if (type == DICEGPU_QUADRATIC_SF) {
      N = 12;
      // Quadratic_Shape_Function ctor deltas (:481-492)
      const float d[12] = {0.001f, 0.001f, 1.0e-6f, 1.0e-6f, 1.0e-6f, 1.0f,
                           0.001f, 0.001f, 1.0e-6f, 1.0e-6f, 1.0e-6f, 1.0f};
      for (int i = 0; i < 12; ++i) { deltas[i] = d[i]; p[i] = 0.0f; }
      p[0] = 1.0f;  // QUAD_A
      p[7] = 1.0f;  // QUAD_H
      return;
    }
    int k = 2;
    iu = 0; iv = 1; it = iex = iey = ig = -1;
    if (P.enable_rotation) it = k++;
    if (P.enable_normal_strain) { iex = k++; iey = k++; }
    if (P.enable_shear_strain) ig = k++;
    N = k;
    for (int i = 0; i < N; ++i) { p[i] = 0.0f; deltas[i] = (float)P.robust_delta_theta; }
    deltas[iu] = (float)P.robust_delta_disp;
    deltas[iv] = (float)P.robust_delta_disp;
  }

  // Affine_Shape_Function::map (:220-248) / Quadratic_Shape_Function::map (:509-520)
  void map(float x, float y, float cx, float cy, float& ox, float& oy) const {
    const float dx = x - cx, dy = y - cy;
    if (type == DICEGPU_QUADRATIC_SF) {
      ox = p[0] * dx + p[1] * dy + p[2] * dx * dy + p[3] * dx * dx + p[4] * dy * dy + p[5] + cx;
      oy = p[6] * dx + p[7] * dy + p[8] * dx * dy + p[9] * dx * dx + p[10] * dy * dy + p[11] + cy;
      return;
    }
    const float theta = it >= 0 ? p[it] : 0.0f;
    const float dudx = iex >= 0 ? p[iex] : 0.0f;
    const float dvdy = iey >= 0 ? p[iey] : 0.0f;
    const float gxy = ig >= 0 ? p[ig] : 0.0f;
    const float cost = cos_f(theta), sint = sin_f(theta);
    const float Dx = (float)((1.0 + dudx) * dx + gxy * dy);
    const float Dy = (float)((1.0 + dvdy) * dy + gxy * dx);
    ox = cost * Dx - sint * Dy + p[iu] + cx;
    oy = sint * Dx + cost * Dy + p[iv] + cy;
  }

  // map_to_u_v_theta (affine :333-347; quadratic :552-578)
  void map_to_u_v_theta(float cx, float cy, float& u, float& v, float& t) const {
    if (type == DICEGPU_QUADRATIC_SF) {
      float cxp, cyp, rxp, ryp;
      map(cx, cy, cx, cy, cxp, cyp);
      u = cxp - cx;
      v = cyp - cy;
      map((float)(cx + 5.0), cy, cx, cy, rxp, ryp);
      const float ax = rxp - cxp, ay = ryp - cyp;
      const float mag_a = std::sqrt(ax * ax + ay * ay);
      const float bx = 5.0f, by = 0.0f, mag_b = 5.0f;
      const float adb = (ax * bx + ay * by) / (mag_a * mag_b);
      t = ay < 0.0f ? (float)(kTwoPi - (double)acos_f(adb)) : acos_f(adb);
      return;
    }
    u = p[iu];
    v = p[iv];
    t = it >= 0 ? p[it] : 0.0f;
  }

  // residuals (affine :350-396, quadratic :580-614)
  void residuals(float x, float y, float cx, float cy, float gx, float gy, float* r,
                 bool use_ref_grads) const {
    if (type == DICEGPU_QUADRATIC_SF) {
      const float dx = x - cx, dy = y - cy;
      float Gx = gx, Gy = gy;
      if (use_ref_grads) {
        float u, v, th;
        map_to_u_v_theta(cx, cy, u, v, th);
        const float c = cos_f(th), s = sin_f(th);
        Gx = c * gx - s * gy;
        Gy = s * gx + c * gy;
      }
      r[0] = Gx * dx; r[1] = Gx * dy; r[2] = Gx * dx * dy; r[3] = Gx * dx * dx;
      r[4] = Gx * dy * dy; r[5] = Gx;
      r[6] = Gy * dx; r[7] = Gy * dy; r[8] = Gy * dx * dy; r[9] = Gy * dx * dx;
      r[10] = Gy * dy * dy; r[11] = Gy;
      return;
    }
    const float theta = it >= 0 ? p[it] : 0.0f;
    const float dudx = iex >= 0 ? p[iex] : 0.0f;
    const float dvdy = iey >= 0 ? p[iey] : 0.0f;
    const float gxy = ig >= 0 ? p[ig] : 0.0f;
    const float c = cos_f(theta), s = sin_f(theta);
    const float dx = x - cx, dy = y - cy;
    const float Dx = (float)((1.0 + dudx) * dx + gxy * dy);
    const float Dy = (float)((1.0 + dvdy) * dy + gxy * dx);
    const float Gx = use_ref_grads ? c * gx - s * gy : gx;
    const float Gy = use_ref_grads ? s * gx + c * gy : gy;
    r[iu] = Gx;
    r[iv] = Gy;
    if (it >= 0) r[it] = Gx * (-s * Dx - c * Dy) + Gy * (c * Dx - s * Dy);
    if (iex >= 0) r[iex] = Gx * dx * c + Gy * dx * s;
    if (iey >= 0) r[iey] = -Gx * dy * s + Gy * dy * c;
    if (ig >= 0) r[ig] = Gx * (c * dy - s * dx) + Gy * (s * dy + c * dx);
  }

  // test_for_convergence (base :91-102 for quadratic; affine :433-459)
  bool converged(const float* old, float tol) const {
    bool conv = true;
    if (type == DICEGPU_QUADRATIC_SF) {
      for (int i = 0; i < N; ++i)
        if (std::abs(p[i] - old[i]) >= tol) conv = false;
      return conv;
    }
    if (std::abs(p[iu] - old[iu]) >= tol) conv = false;
    if (std::abs(p[iv] - old[iv]) >= tol) conv = false;
    if (it >= 0 && std::abs(p[it] - old[it]) >= tol) conv = false;
    return conv;
  }

  // initialize_parameters_from_fields (affine :252-312, DISPLACEMENT_BASED
  // projection; quadratic through the base class, :125-137)
  void from_fields(const double* f) {
    if (type == DICEGPU_QUADRATIC_SF) {
      for (int i = 0; i < 12; ++i) p[i] = (float)f[DICEGPU_F_QUAD_A + i];
      return;
    }
    p[iu] = (float)f[DICEGPU_F_DISP_X];
    p[iv] = (float)f[DICEGPU_F_DISP_Y];
    if (it >= 0) p[it] = (float)f[DICEGPU_F_ROT_Z];
    if (iex >= 0) p[iex] = (float)f[DICEGPU_F_STRETCH_XX];
    if (iey >= 0) p[iey] = (float)f[DICEGPU_F_STRETCH_YY];
    if (ig >= 0) p[ig] = (float)f[DICEGPU_F_SHEAR_XY];
  }

  // save_fields (base :65-74; quadratic :616-629 also stores u, v, theta)
  void to_fields(double* f, float cx, float cy) const {
    if (type == DICEGPU_QUADRATIC_SF) {
      for (int i = 0; i < 12; ++i) f[DICEGPU_F_QUAD_A + i] = p[i];
      float u, v, t;
      map_to_u_v_theta(cx, cy, u, v, t);
      f[DICEGPU_F_DISP_X] = u;
      f[DICEGPU_F_DISP_Y] = v;
      f[DICEGPU_F_ROT_Z] = t;
      return;
    }
    f[DICEGPU_F_DISP_X] = p[iu];
    f[DICEGPU_F_DISP_Y] = p[iv];
    if (it >= 0) f[DICEGPU_F_ROT_Z] = p[it];
    if (iex >= 0) f[DICEGPU_F_STRETCH_XX] = p[iex];
    if (iey >= 0) f[DICEGPU_F_STRETCH_YY] = p[iey];
    if (ig >= 0) f[DICEGPU_F_SHEAR_XY] = p[ig];
  }
};

// ---------------------------------------------------------------------------
// Subset (DICe_Subset.cpp)
// ---------------------------------------------------------------------------
typedef std::set<std::pair<int, int>> PixelSet;   // (y, x), as the reference stores them

struct Subset {
  int cx = 0, cy = 0, npix = 0;
  std::vector<int> x, y;
  std::vector<float> ref, def, gx, gy;
  std::vector<char> active, deact;
  bool has_gradients = false;
  const PixelSet* obstructed = nullptr;   // obstructed_coords_
  const PixelSet* blocked = nullptr;      // pixels_blocked_by_other_subsets_
  // subset evolution (turn_on_previously_obstructed_pixels): per pixel 1
  // active, 0 inactive (excluded), 2 turned on with the stored intensity
  uint8_t* flag = nullptr;
  float* fstore = nullptr;

  // Subset(cx,cy,w,h) (:78-113): odd extent, negative coordinates clamped to 0.
  void init_square(int cx_, int cy_, int size) {
    cx = cx_; cy = cy_;
    const int hw = size / 2;
    npix = (2 * hw + 1) * (2 * hw + 1);
    x.resize(npix); y.resize(npix);
    int k = 0;
    for (int yy = cy - hw; yy <= cy + hw; ++yy)
      for (int xx = cx - hw; xx <= cx + hw; ++xx) {
        x[k] = xx < 0 ? 0 : xx;
        y[k] = yy < 0 ? 0 : yy;
        ++k;
      }
    alloc();
  }
  // Subset(cx,cy,x[],y[]) (:49-76)
  void init_list(int cx_, int cy_, const int32_t* px, const int32_t* py, int n) {
    cx = cx_; cy = cy_; npix = n;
    x.resize(n); y.resize(n);
    for (int i = 0; i < n; ++i) {
      x[i] = px[i] < 0 ? 0 : px[i];
      y[i] = py[i] < 0 ? 0 : py[i];
    }
    alloc();
  }
  void alloc() {
    ref.assign(npix, 0.0f); def.assign(npix, 0.0f);
    gx.assign(npix, 0.0f); gy.assign(npix, 0.0f);
    active.assign(npix, 1); deact.assign(npix, 0);
  }
  // initialize(ref_img) with no shape function (:385-389, :428-437)
  void init_ref(const Image& im) {
    for (int i = 0; i < npix; ++i) ref[i] = im.at(im.I, (long)y[i] * im.w + x[i]);
    if (flag)
      for (int i = 0; i < npix; ++i) {
        active[i] = flag[i] != 0;
        if (flag[i] == 2) ref[i] = fstore[i];
      }
    if (im.has_gradients) {
      for (int i = 0; i < npix; ++i) {
        gx[i] = im.at(im.gx, (long)y[i] * im.w + x[i]);
        gy[i] = im.at(im.gy, (long)y[i] * im.w + x[i]);
      }
      has_gradients = true;
    }
  }
  // initialize(def_img, DEF_INTENSITIES, shape_function, interp) (:390-426)
  void init_def(const Image& im, const ShapeFn& sf, int interp) {
    const float fcx = (float)cx, fcy = (float)cy;
    for (int i = 0; i < npix; ++i) {
      float mx, my;
      sf.map((float)x[i], (float)y[i], fcx, fcy, mx, my);
      const int px = ((int)(mx + 0.5) == (int)(mx)) ? (int)(mx) : (int)(mx) + 1;
      const int py = ((int)(my + 0.5) == (int)(my)) ? (int)(my) : (int)(my) + 1;
      if (px < 4 || px >= im.w - 4 || py < 4 || py >= im.h - 4) {
        deact[i] = 1;
        continue;
      }
      // is_obstructed_pixel (:446-460) with its own rounding of the position
      if (obstructed && !obstructed->empty()) {
        int c_x = (int)mx;
        if (mx - (float)(int)mx >= 0.5) c_x++;
        int c_y = (int)my;
        if (my - (float)(int)my >= 0.5) c_y++;
        if (obstructed->count(std::make_pair(c_y, c_x))) {
          deact[i] = 1;
          continue;
        }
      }
      if (blocked && !blocked->empty() && blocked->count(std::make_pair(py, px))) {
        deact[i] = 1;
        continue;
      }
      deact[i] = 0;
      interpolate(im, interp, def[i], gx[i], gy[i], im.has_gradients, mx - 0.0f, my - 0.0f);
    }
  }
  int num_active() const {
    int n = 0;
    for (int i = 0; i < npix; ++i) if (active[i] && !deact[i]) ++n;
    return n;
  }
  // mean (:285-301)
  float mean(bool def_target) const {
    float m = 0.0f;
    const int na = num_active();
    const std::vector<float>& v = def_target ? def : ref;
    for (int i = 0; i < npix; ++i) if (active[i] && !deact[i]) m += v[i];
    return na != 0 ? m / na : 0.0f;
  }
  // mean with sum (:303-321)
  float mean(bool def_target, float& sum) const {
    const float m = mean(def_target);
    const std::vector<float>& v = def_target ? def : ref;
    sum = 0.0f;
    for (int i = 0; i < npix; ++i)
      if (active[i] && !deact[i]) sum += (v[i] - m) * (v[i] - m);
    sum = std::sqrt(sum);
    return m;
  }
  // gamma (:323-340)
  float gamma() const {
    float sr = 0.0f, sd = 0.0f;
    const float mr = mean(false, sr);
    const float md = mean(true, sd);
    if (sr == 0.0f || sd == 0.0f) return -1.0f;
    float g = 0.0f;
    for (int i = 0; i < npix; ++i)
      if (active[i] && !deact[i]) {
        const float val = (def[i] - md) / sd - (ref[i] - mr) / sr;
        g += val * val;
      }
    return g;
  }
  // contrast_std_dev (:607-620)
  float contrast_std_dev() const {
    const float m = mean(true);
    float sd = 0.0f;
    int na = 0;
    for (int i = 0; i < npix; ++i)
      if (active[i] && !deact[i]) { ++na; sd += (def[i] - m) * (def[i] - m); }
    return na == 0 ? 0.0f : std::sqrt(sd / na);
  }
  // noise_std_dev (:622-703) on the deformed image
  float noise_std_dev(const Image& im, const ShapeFn& sf) const {
    static const float mask[3][3] = {{1, -2, 1}, {-2, 4, -2}, {1, -2, 1}};
    int min_x = cx, max_x = cx, min_y = cy, max_y = cy, ndeact = 0;
    for (int i = 0; i < npix; ++i) {
      if (deact[i] || !active[i]) { ++ndeact; continue; }
      if (x[i] < min_x) min_x = x[i];
      if (x[i] > max_x) max_x = x[i];
      if (y[i] < min_y) min_y = y[i];
      if (y[i] > max_y) max_y = y[i];
    }
    if (ndeact == npix) return -1.0f;
    float u, v, t;
    sf.map_to_u_v_theta((float)cx, (float)cy, u, v, t);
    min_x = (int)(min_x + u); max_x = (int)(max_x + u);
    min_y = (int)(min_y + v); max_y = (int)(max_y + v);
    const int img_h = im.h, img_w = im.w;
    if (min_x < 0) min_x = 0;
    if (min_y < 0) min_y = 0;
    if (max_x >= img_w) min_x = 0;  // the reference resets min_x here (:667)
    if (max_y >= img_h) min_y = 0;  // and min_y here (:668)
    int hh = max_y - min_y + 1, ww = max_x - min_x + 1;
    if (ww < 3) ww = 3;
    if (hh < 3) hh = 3;
    float variance = 0.0f;
    for (int yy = min_y; yy < max_y; ++yy) {
      for (int xx = min_x; xx < max_x; ++xx) {
        if (xx < 1 || xx >= img_w - 1 || yy < 1 || yy >= img_h - 1) {
          const float a = im.at(im.I, (long)yy * img_w + xx);
          variance += std::sqrt(a * a);
        } else {
          float conv = 0.0f;
          for (int j = 0; j < 3; ++j)
            for (int i = 0; i < 3; ++i)
              conv += im.I[(long)(yy + j - 1) * img_w + xx + i - 1] * mask[i][j];
          variance += std::abs(conv);
        }
      }
    }
    variance = (float)(variance * (std::sqrt(0.5 * kPi) / (6.0 * (ww - 2) * (hh - 2))));
    return variance;
  }
};

// ---------------------------------------------------------------------------
// LU factorisation + inverse standing in for LAPACK DGETRF/DGETRI
// (DICe_Objective.cpp:571, 591).  Partial pivoting on the first maximal
// |a_ij| (IDAMAX), column scaling by the reciprocal pivot, rank-1 trailing
// update (the unblocked DGETF2 order).  A zero pivot leaves the column
// unscaled and records info; DGETRI then returns early and leaves the LU
// factors in place, which the reference goes on to use as the "inverse".
// ---------------------------------------------------------------------------
static int lu_factor(double* A, int N, int* piv) {  // row-major A[i*N+j]
  int info = 0;
  for (int j = 0; j < N; ++j) {
    int p = j;
    double best = std::abs(A[j * N + j]);
    for (int i = j + 1; i < N; ++i)
      if (std::abs(A[i * N + j]) > best) { best = std::abs(A[i * N + j]); p = i; }
    piv[j] = p;
    if (A[p * N + j] != 0.0) {
      if (p != j)
        for (int k = 0; k < N; ++k) std::swap(A[j * N + k], A[p * N + k]);
      const double r = 1.0 / A[j * N + j];
      for (int i = j + 1; i < N; ++i) A[i * N + j] *= r;
    } else if (info == 0) {
      info = j + 1;
    }
    for (int i = j + 1; i < N; ++i)
      for (int k = j + 1; k < N; ++k) A[i * N + k] -= A[i * N + j] * A[j * N + k];
  }
  return info;
}

static void lu_inverse(const double* LU, const int* piv, int N, double* inv) {
  // columns of inv(A) solve A x = e_k: x = U^-1 L^-1 P e_k
  std::vector<double> col(N);
  for (int k = 0; k < N; ++k) {
    for (int i = 0; i < N; ++i) col[i] = (i == k) ? 1.0 : 0.0;
    for (int j = 0; j < N; ++j)
      if (piv[j] != j) std::swap(col[j], col[piv[j]]);
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < i; ++j) col[i] -= LU[i * N + j] * col[j];
    for (int i = N - 1; i >= 0; --i) {
      for (int j = i + 1; j < N; ++j) col[i] -= LU[i * N + j] * col[j];
      col[i] /= LU[i * N + i];
    }
    for (int i = 0; i < N; ++i) inv[i * N + k] = col[i];
  }
}

// ---------------------------------------------------------------------------
// Objective (DICe_Objective.cpp) + simplex (DICe_Simplex.cpp)
// ---------------------------------------------------------------------------
struct Ctx {
  dicegpu_params P;
  Image ref, def;
};

// Per-subset side outputs: work counters, and where the uncertainty fields of
// a converged Gauss-Newton solve go (nullptr: not requested).
struct Counters {
  int gn_iters = 0;
  int simplex_evals = 0;
  double* unc = nullptr;
  float ucx = 0.0f, ucy = 0.0f;   // the subset's COORD_X / COORD_Y fields
};

// Image_::interpolate_bilinear (DICe_Image.cpp:432-445), intensity only.
static float bilinear_intensity(const Image& im, float lx, float ly) {
  if (!(lx >= 0.0f && lx < im.w - 1.5 && ly >= 0.0f && ly < im.h - 1.5)) return 0.0f;   // NaN too
  const int x1 = (int)lx, x2 = x1 + 1, y1 = (int)ly, y2 = y1 + 1;
  return im.I[(long)y1 * im.w + x1] * (x2 - lx) * (y2 - ly) +
         im.I[(long)y1 * im.w + x2] * (lx - x1) * (y2 - ly) +
         im.I[(long)y2 * im.w + x2] * (lx - x1) * (ly - y1) +
         im.I[(long)y2 * im.w + x1] * (x2 - lx) * (ly - y1);
}

// Image_::interpolate_keys_fourth (DICe_Image.cpp:890-924), intensity only:
// unlike the _all variant it returns the bilinear value near the border.
static float keys_intensity(const Image& im, float lx, float ly) {
  if (!(lx > 2.5 && lx < im.w - 3.5 && ly > 2.5 && ly < im.h - 3.5)) return bilinear_intensity(im, lx, ly);
  const int ix = (int)lx, iy = (int)ly;
  const float dx = lx - ix, dy = ly - iy;
  float cx[6], cy[6];
  cx[0] = keys_f2((float)(dx + 2.0));
  cx[1] = keys_f1((float)(dx + 1.0));
  cx[2] = keys_f0(dx);
  cx[3] = keys_f0((float)(1.0 - dx));
  cx[4] = keys_f1((float)(2.0 - dx));
  cx[5] = keys_f2((float)(3.0 - dx));
  cy[0] = keys_f2((float)(dy + 2.0));
  cy[1] = keys_f1((float)(dy + 1.0));
  cy[2] = keys_f0(dy);
  cy[3] = keys_f0((float)(1.0 - dy));
  cy[4] = keys_f1((float)(2.0 - dy));
  cy[5] = keys_f2((float)(3.0 - dy));
  float v = 0.0f;
  for (int m = 0; m < 6; ++m)
    for (int n = 0; n < 6; ++n) v += cy[m] * cx[n] * im.I[(long)(iy - 2 + m) * im.w + ix - 2 + n];
  return v;
}

// Objective::gamma (:58-76)
static float objective_gamma(const Ctx& C, Subset& s, const ShapeFn& sf, Counters* cnt) {
  s.init_def(C.def, sf, C.P.interpolation);
  if (cnt) cnt->simplex_evals++;
  float g = s.gamma();
  if (C.P.normalize_gamma_with_active_pixels) {
    int na = 0;
    for (int i = 0; i < s.npix; ++i) if (s.active[i]) ++na;
    // gamma /= (num_active==0.0 ? 1.0 : num_active): a double divisor (:70-71)
    if (na > 0) g = (float)(g / (double)na);
  }
  return g;
}

// Objective::sigma (:150-184)
static float objective_sigma(const Ctx& C, const Subset& s, const ShapeFn& sf, float& noise) {
  if (!s.has_gradients) return 0.0f;
  noise = s.noise_std_dev(C.def, sf);
  if (noise < 0.0f) return -1.0f;
  float sgx = 0.0f, sgy = 0.0f;
  for (int i = 0; i < s.npix; ++i) {
    if (!s.active[i] || s.deact[i]) continue;
    sgx += s.gx[i] * s.gx[i];
    sgy += s.gy[i] * s.gy[i];
  }
  const float sg = sgx > sgy ? sgy : sgx;
  return sg > 0.0f ? (float)std::sqrt(2.0 * noise * noise / sg) : -1.0f;
}

// Objective::computeUncertaintyFields (DICe_Objective.cpp:193-299) without an
// image deformer, so the exact motion (bx, by) is zero: FIELD_1..FIELD_7 go to
// out[0..6].  Every pixel of the subset takes part, active or not, with the
// gradients the last deformed-state initialisation left in the subset; u, v
// are the converged parameters mapped at the subset's coordinates.  All sums
// are float; the field store rounds to float as DICe's float fields do.
static void uncertainty_fields(const Ctx& C, const Subset& s, const ShapeFn& sf, float fcx,
                               float fcy, double* out) {
  float u, v, t;
  sf.map_to_u_v_theta(fcx, fcy, u, v, t);
  float norm_uhat_2 = 0.0f, uhat_dot_g = 0.0f, err_dot_g = 0.0f, err_dot_jg = 0.0f, int_r = 0.0f;
  float sssig = 1.0f;
  for (int i = 0; i < s.npix; ++i) {
    const float x = (float)s.x[i], y = (float)s.y[i];
    const float gx = s.gx[i], gy = s.gy[i];
    sssig += gx * gx + gy * gy;
    norm_uhat_2 += u * u + v * v;
    const float g2 = gx * gx + gy * gy;
    const float inv_g2 = g2 < 1.0e-4 ? 0.0f : (float)(1.0 / g2);
    const float a = u * gx + v * gy;
    uhat_dot_g += a * a * inv_g2;
    err_dot_g += a * a * inv_g2;
    const float j = v * gx - u * gy;
    err_dot_jg += j * j * inv_g2;
    const float r0 = C.ref.at(C.ref.I, (long)s.y[i] * C.ref.w + s.x[i]);
    const float sub_r = keys_intensity(C.def, x + u, y + v) - r0;
    const float sub_r_exact = keys_intensity(C.def, x + 0.0f, y + 0.0f) - r0;
    int_r += (sub_r - sub_r_exact) * (sub_r - sub_r_exact) * inv_g2;
  }
  sssig = (float)(sssig / (s.npix == 0 ? 1.0 : (double)s.npix));
  const float cos_hat = norm_uhat_2 == 0.0f ? 1.0f : std::sqrt(uhat_dot_g / norm_uhat_2);
  out[0] = cos_hat;
  out[1] = 1.0;
  out[2] = std::sqrt(err_dot_g + err_dot_jg);
  out[3] = (float)(cos_hat == 0.0f ? 0.0 : 1.0 / (double)cos_hat * (double)std::sqrt(int_r));
  out[4] = std::sqrt(err_dot_g);
  out[5] = std::sqrt(int_r);
  out[6] = sssig;
}

// Objective_ZNSSD::computeUpdateFast (:430-657)
static int compute_update_fast(const Ctx& C, Subset& s, ShapeFn& sf, int& num_iterations,
                               double* cond_out, Counters* cnt) {
  const int N = sf.N;
  const float tol = (float)C.P.fast_solver_tolerance;
  const int max_its = C.P.max_solver_iterations_fast;
  const bool use_ref_grads = !C.def.has_gradients;
  double H[144], q[12], Hinv[144];
  float r[12], def_old[12], def_update[12], def_update_old[12];
  int piv[12];
  for (int i = 0; i < N; ++i) def_update_old[i] = 0.0f;
  const float fcx = (float)s.cx, fcy = (float)s.cy;
  const float meanF = s.mean(false);
  int solve_it = 0;
  for (; solve_it <= max_its; ++solve_it) {
    num_iterations = solve_it;
    s.init_def(C.def, sf, C.P.interpolation);
    if (cnt) cnt->gn_iters++;
#ifdef ORACLE_DEF_MEAN_FP64
    // sensitivity variant (not the reference): the deformed mean summed in
    // double, the rounding a compiler or library change could also bring
    float meanG = 0.0f;
    {
      double m = 0.0;
      int na = 0;
      for (int i = 0; i < s.npix; ++i)
        if (s.active[i] && !s.deact[i]) { m += s.def[i]; ++na; }
      meanG = na ? (float)(m / na) : 0.0f;
    }
#else
    const float meanG = s.mean(true);
#endif
    for (int i = 0; i < N * N; ++i) H[i] = 0.0;
    for (int i = 0; i < N; ++i) q[i] = 0.0;
    for (int idx = 0; idx < s.npix; ++idx) {
      if (s.deact[idx] || !s.active[idx]) continue;
      const float GmF = (s.def[idx] - meanG) - (s.ref[idx] - meanF);
      for (int i = 0; i < N; ++i) r[i] = 0.0f;
      sf.residuals((float)s.x[idx], (float)s.y[idx], fcx, fcy, s.gx[idx], s.gy[idx], r,
                   use_ref_grads);
      for (int i = 0; i < N; ++i) {
        q[i] += GmF * r[i];
        for (int j = 0; j < N; ++j) H[i * N + j] += r[i] * r[j];
      }
    }
    if (C.P.levenberg_marquardt_regularization_factor > 0.0) {
      const float alpha = (float)C.P.levenberg_marquardt_regularization_factor;
      H[0] += alpha;
      H[1 * N + 1] += alpha;
    }
    const float det_h = (float)(H[0] * H[N + 1] - H[N] * H[1]);
    const double nsq = H[0] * H[0] + H[1] * H[1] + H[N] * H[N] + H[N + 1] * H[N + 1];
    const float norm_H = (float)std::sqrt(nsq);
    float cond = -1.0f;
    if (det_h != 0.0f) {
      const float norm_Hi = (float)std::sqrt((1.0 / (double)(det_h * det_h)) * nsq);
      cond = norm_H * norm_Hi;
    }
    const int info = lu_factor(H, N, piv);
    if (cond_out) *cond_out = cond;
    if (cond > 1.0e12f) return DICEGPU_HESSIAN_SINGULAR;
    const double* M = H;
    if (info == 0) {
      lu_inverse(H, piv, N, Hinv);
      M = Hinv;
    }
    for (int i = 0; i < N; ++i) def_old[i] = sf.p[i];
    for (int i = 0; i < N; ++i) def_update[i] = 0.0f;
    for (int i = 0; i < N; ++i)
      for (int j = 0; j < N; ++j) def_update[i] += M[i * N + j] * (-1.0) * q[j];
    if (C.P.momentum_factor != 0.0) {
      const float mom = (float)C.P.momentum_factor;
      for (int i = 0; i < N; ++i) {
        def_update[i] += mom * def_update_old[i];
        def_update_old[i] = def_update[i];
      }
    }
    for (int i = 0; i < N; ++i) sf.p[i] += def_update[i];
    if (sf.converged(def_old, tol)) {
      if (cnt && cnt->unc) uncertainty_fields(C, s, sf, cnt->ucx, cnt->ucy, cnt->unc);
      break;
    }
  }
  if (solve_it > max_its) return DICEGPU_MAX_ITERATIONS_REACHED;
  return DICEGPU_CORRELATION_SUCCESSFUL;
}

// Simplex::minimize (DICe_Simplex.cpp:60-277) via Subset_Simplex::objective
// (:298-302).  `last_eval` receives the parameters of the last evaluation (the
// subset's deformed state belongs to that point).
static int simplex_minimize(const Ctx& C, Subset& s, ShapeFn& sf, int& num_iterations,
                            float threshold, Counters* cnt) {
  const int nd = sf.N;
  const int max_iterations = C.P.max_solver_iterations_robust;
  const double tolerance = C.P.robust_solver_tolerance;
  const float tiny = 1.0e-10f;
  float* vars = sf.p;  // the variables alias the shape-function parameters
  float init_vars[12];
  for (int i = 0; i < nd; ++i) init_vars[i] = vars[i];
  const int mpts = nd + 1;
  float gv[13];
  float pts[13][12];
  for (int i = 0; i < mpts; ++i) {
    for (int j = 0; j < nd; ++j) pts[i][j] = vars[j];
    if (i > 0) pts[i][i - 1] += sf.deltas[i - 1];
    for (int j = 0; j < nd; ++j) vars[j] = pts[i][j];
    gv[i] = objective_gamma(C, s, sf, cnt);
    if (i == 0 && gv[i] < threshold && gv[i] >= 0.0f) {
      num_iterations = 0;
      return DICEGPU_CORRELATION_SUCCESSFUL;
    }
    for (int j = 0; j < nd; ++j) vars[j] = init_vars[j];
  }
  int inhi = 0;
  float ysave;
  float psum[12], ptry[12];
  for (int j = 0; j < nd; ++j) {
    float sum = 0.0f;
    for (int i = 0; i < mpts; ++i) sum += pts[i][j];
    psum[j] = sum;
  }
  float old_rtol = 0.0f, gamma_new = 0.0f, gamma_old = -1.0f;
  int gamma_repeats = 0;
  const int gamma_repeats_allowed = 15;
  const float gamma_tol = 1.0e-8f;
  int iteration = 0;
  for (iteration = 0; iteration < max_iterations; iteration++) {
    if (iteration >= max_iterations - 1) {
      num_iterations = iteration;
      return DICEGPU_MAX_ITERATIONS_REACHED;
    }
    int ilo = 0;
    int ihi = gv[0] > gv[1] ? (inhi = 1, 0) : (inhi = 0, 1);
    for (int i = 0; i < mpts; i++) {
      if (gv[i] <= gv[ilo]) ilo = i;
      if (gv[i] > gv[ihi]) {
        inhi = ihi;
        ihi = i;
      } else if (gv[i] > gv[inhi] && i != ihi)
        inhi = i;
    }
    const float rtol = (float)(2.0 * std::abs(gv[ihi] - gv[ilo]) /
                               (std::abs(gv[ihi]) + std::abs(gv[ilo]) + tiny));
    const float rtol_diff = std::abs(rtol - old_rtol);
    old_rtol = rtol;
    if (std::abs(gamma_new - gamma_old) < gamma_tol) gamma_repeats++;
    gamma_old = gamma_new;
    if (rtol < tolerance || rtol_diff < tolerance || gamma_repeats > gamma_repeats_allowed) {
      std::swap(gv[0], gv[ilo]);
      for (int i = 0; i < nd; i++) std::swap(pts[0][i], pts[ilo][i]);
      break;
    }
    float ytry, fac, fac1, fac2;
    fac = -1.0f;
    fac1 = (float)((1.0 - fac) / nd);
    fac2 = fac1 - fac;
    for (int j = 0; j < nd; j++) ptry[j] = psum[j] * fac1 - pts[ihi][j] * fac2;
    for (int n = 0; n < nd; ++n) vars[n] = ptry[n];
    ytry = objective_gamma(C, s, sf, cnt);
    if (ytry < gv[ihi]) {
      gv[ihi] = ytry;
      for (int j = 0; j < nd; j++) {
        psum[j] += ptry[j] - pts[ihi][j];
        pts[ihi][j] = ptry[j];
      }
    }
    if (ytry <= gv[ilo]) {
      fac = 2.0f;
      fac1 = (float)((1.0 - fac) / nd);
      fac2 = fac1 - fac;
      for (int j = 0; j < nd; j++) ptry[j] = psum[j] * fac1 - pts[ihi][j] * fac2;
      for (int n = 0; n < nd; ++n) vars[n] = ptry[n];
      ytry = objective_gamma(C, s, sf, cnt);
      if (ytry < gv[ihi]) {
        gv[ihi] = ytry;
        for (int j = 0; j < nd; j++) {
          psum[j] += ptry[j] - pts[ihi][j];
          pts[ihi][j] = ptry[j];
        }
      }
    } else if (ytry >= gv[inhi]) {
      ysave = gv[ihi];
      fac = 0.5f;
      fac1 = (float)((1.0 - fac) / nd);
      fac2 = fac1 - fac;
      for (int j = 0; j < nd; j++) ptry[j] = psum[j] * fac1 - pts[ihi][j] * fac2;
      for (int n = 0; n < nd; ++n) vars[n] = ptry[n];
      ytry = objective_gamma(C, s, sf, cnt);
      if (ytry < gv[ihi]) {
        gv[ihi] = ytry;
        for (int j = 0; j < nd; j++) {
          psum[j] += ptry[j] - pts[ihi][j];
          pts[ihi][j] = ptry[j];
        }
      }
      if (ytry >= ysave) {
        for (int i = 0; i < mpts; i++) {
          if (i != ilo) {
            for (int j = 0; j < nd; j++)
              pts[i][j] = psum[j] = (float)(0.5 * (pts[i][j] + pts[ilo][j]));
            for (int n = 0; n < nd; ++n) vars[n] = psum[n];
            gv[i] = objective_gamma(C, s, sf, cnt);
          }
        }
        for (int j = 0; j < nd; j++) {
          float sum = 0.0f;
          for (int i = 0; i < mpts; i++) sum += pts[i][j];
          psum[j] = sum;
        }
      }
    }
    gamma_new = objective_gamma(C, s, sf, cnt);
  }
  num_iterations = iteration;
  return DICEGPU_CORRELATION_SUCCESSFUL;
}

// Objective::computeUpdateRobust (:369-388)
static int compute_update_robust(const Ctx& C, Subset& s, ShapeFn& sf, int& num_iterations,
                                 Counters* cnt) {
  return simplex_minimize(C, s, sf, num_iterations, (float)C.P.skip_solve_gamma_threshold, cnt);
}

// Schema::record_failed_step (DICe_Schema.cpp:1959-1983)
static void record_failed_step(double* f, int status, int num_iterations) {
  f[DICEGPU_F_SIGMA] = -1.0;
  f[DICEGPU_F_MATCH] = -1.0;
  f[DICEGPU_F_GAMMA] = -1.0;
  f[DICEGPU_F_BETA] = -1.0;
  f[DICEGPU_F_OMEGA] = -1.0;
  f[DICEGPU_F_NOISE] = -1.0;
  f[DICEGPU_F_CONTRAST] = -1.0;
  f[DICEGPU_F_ACTIVE_PIXELS] = -1.0;
  f[DICEGPU_F_STATUS] = status;
  f[DICEGPU_F_ITERATIONS] = num_iterations;
}

// Field_Value_Initializer::initial_guess (DICe_Initializer.cpp:398-436), own id.
// Field_Value_Initializer::initial_guess (DICe_Initializer.cpp:398-436):
// the subset's own field row, or its neighbour's (nf) with neighbour
// initialization; the quadratic parameters then move to this subset's
// centroid (Quadratic_Shape_Function::update_params_for_centroid_change,
// DICe_LocalShapeFunction.cpp:632-651, float parameters, the 2.0 literals
// in double).
static int initial_guess(const double* f, const double* nf, ShapeFn& sf) {
  const double* g = nf ? nf : f;
  if (g[DICEGPU_F_SIGMA] == -1.0) return DICEGPU_INITIALIZE_FAILED;
  sf.from_fields(g);
  if (!nf) return DICEGPU_INITIALIZE_USING_PREVIOUS_FRAME_SUCCESSFUL;
  if (sf.type == DICEGPU_QUADRATIC_SF) {
    const float dx = (float)f[DICEGPU_F_COORD_X] - (float)nf[DICEGPU_F_COORD_X];
    const float dy = (float)f[DICEGPU_F_COORD_Y] - (float)nf[DICEGPU_F_COORD_Y];
    float* q = sf.p;
    const float A = q[0], B = q[1], C = q[2], D = q[3], E = q[4];
    const float G = q[6], H = q[7], I = q[8], J = q[9], K = q[10];
    q[0] = (float)((double)q[0] + ((double)(C * dy) + 2.0 * D * dx));
    q[1] = (float)((double)q[1] + ((double)(C * dx) + 2.0 * E * dy));
    q[5] += A * dx + B * dy + C * dx * dy + D * dx * dx + E * dy * dy - dx;
    q[6] = (float)((double)q[6] + ((double)(I * dy) + 2.0 * J * dx));
    q[7] = (float)((double)q[7] + ((double)(I * dx) + 2.0 * K * dy));
    q[11] += G * dx + H * dy + I * dx * dy + J * dx * dx + K * dy * dy - dy;
  }
  return DICEGPU_INITIALIZE_USING_NEIGHBOR_VALUE_SUCCESSFUL;
}

// Objective::beta (DICe_Objective.cpp:78-148): finite-difference slope of gamma
// in u, v (and theta when rotation is enabled), unnormalised.
static float objective_beta(const Ctx& C, Subset& s, const ShapeFn& sf_in) {
  Ctx C2 = C;
  C2.P.normalize_gamma_with_active_pixels = 0;
  const float eps[3] = {0.1f, 0.1f, 0.1f};
  const float fac[3] = {1.0e-3f, 1.0e-3f, 1.0e-1f};
  const float g0 = objective_gamma(C2, s, sf_in, nullptr);
  float dir[3] = {0.0f, 0.0f, 0.0f};
  const bool rot = C.P.enable_rotation != 0;
  for (int i = 0; i < 3; ++i) {
    ShapeFn t = sf_in;
    float u, v, th;
    t.map_to_u_v_theta((float)s.cx, (float)s.cy, u, v, th);
    if (!rot && i == 2) continue;
    if (i == 0) u += eps[i]; else if (i == 1) v += eps[i]; else th += eps[i];
    auto insert = [&](ShapeFn& sfn) {
      if (sfn.type == DICEGPU_QUADRATIC_SF) {
        for (int k = 0; k < 12; ++k) sfn.p[k] = 0.0f;
        sfn.p[0] = cos_f(th); sfn.p[1] = -sin_f(th);
        sfn.p[6] = sin_f(th); sfn.p[7] = cos_f(th);
        sfn.p[5] = u; sfn.p[11] = v;
      } else {
        sfn.p[sfn.iu] = u; sfn.p[sfn.iv] = v;
        if (sfn.it >= 0) sfn.p[sfn.it] = th;
      }
    };
    insert(t);
    const float gp = objective_gamma(C2, s, t, nullptr);
    if (i == 0) u -= 2 * eps[i]; else if (i == 1) v -= 2 * eps[i]; else th -= 2 * eps[i];
    insert(t);
    const float gm = objective_gamma(C2, s, t, nullptr);
    if (std::abs(gm - g0) < 1.0e-10 || std::abs(gp - g0) < 1.0e-10) {
      objective_gamma(C, s, sf_in, nullptr);
      return -1.0f;
    }
    const float sm = std::abs(eps[i] / (gm - g0)) * fac[i];
    const float sp = std::abs(eps[i] / (gp - g0)) * fac[i];
    dir[i] = (float)((sm + sp) / 2.0);
  }
  float mag = 0.0f;
  for (int i = 0; i < 3; ++i) {
    if (!rot && i == 2) continue;
    mag += dir[i] * dir[i];
  }
  mag = std::sqrt(mag);
  objective_gamma(C, s, sf_in, nullptr);
  return mag;
}

// Schema::generic_correlation_routine (DICe_Schema.cpp:2026-2368) for one subset,
// restricted to the field-value initializer (own or neighbour row, nf) and
// local DIC.
// flags: bit 0 forces the simplex, bit 1 skips the solve (SKIP_SOLVE).
static bool correlate_subset(const Ctx& C, Subset& s, double* f, bool first_frame,
                             unsigned flags, Counters* cnt, const double* nf = nullptr) {
  const bool force_simplex = (flags & 1u) != 0;
  const dicegpu_params& P = C.P;
  if (P.subset_size > 0 && first_frame) {
    const float cur_x = (float)(f[DICEGPU_F_COORD_X] + f[DICEGPU_F_DISP_X]);
    const float cur_y = (float)(f[DICEGPU_F_COORD_Y] + f[DICEGPU_F_DISP_Y]);
    const int hs = P.subset_size / 2;
    if (cur_x < hs || cur_x > C.def.w - hs || cur_y < hs || cur_y > C.def.h - hs) {
      record_failed_step(f, DICEGPU_INITIALIZE_FAILED_BY_EXCEPTION, -1);
      return false;
    }
  }
  int num_iterations = -1;
  ShapeFn sf;
  sf.init(P);
  int init_status = initial_guess(f, nf, sf);
  if (init_status == DICEGPU_INITIALIZE_FAILED) {
    record_failed_step(f, init_status, num_iterations);
    return false;
  }
  // the solve skipped (DICe_Schema.cpp:2118-2143): the initial guess
  // evaluated and recorded as FRAME_SKIPPED
  if ((flags & 2u) || P.skip_all_solves) {
    float noise = 0.0f;
    const float sigma = objective_sigma(C, s, sf, noise);
    const float gamma = objective_gamma(C, s, sf, cnt);
    const float beta = P.output_beta ? objective_beta(C, s, sf) : 0.0f;
    const float contrast = s.contrast_std_dev();
    const int active_pixels = s.num_active();
    sf.to_fields(f, (float)s.cx, (float)s.cy);
    f[DICEGPU_F_SIGMA] = sigma;
    f[DICEGPU_F_MATCH] = 0.0;
    f[DICEGPU_F_GAMMA] = gamma;
    f[DICEGPU_F_BETA] = beta;
    f[DICEGPU_F_NOISE] = noise;
    f[DICEGPU_F_CONTRAST] = contrast;
    f[DICEGPU_F_ACTIVE_PIXELS] = active_pixels;
    f[DICEGPU_F_STATUS] = DICEGPU_FRAME_SKIPPED;
    f[DICEGPU_F_ITERATIONS] = num_iterations;
    return true;
  }
  if (P.initial_gamma_threshold != -1.0) {
    const float g0 = objective_gamma(C, s, sf, cnt);
    if (g0 > P.initial_gamma_threshold || g0 < 0.0f) {
      record_failed_step(f, DICEGPU_INITIALIZE_FAILED, num_iterations);
      return false;
    }
  }
  const float prev_u = (float)f[DICEGPU_F_DISP_X];
  const float prev_v = (float)f[DICEGPU_F_DISP_Y];
  const float prev_t = (float)f[DICEGPU_F_ROT_Z];
  const int opt = P.optimization;
  int corr_status = DICEGPU_CORRELATION_FAILED;
  double cond = 0.0;
  bool cond_set = false;
  if (opt == DICEGPU_SIMPLEX || opt == DICEGPU_SIMPLEX_THEN_GRADIENT_BASED || force_simplex) {
    corr_status = compute_update_robust(C, s, sf, num_iterations, cnt);
  } else {
    corr_status = compute_update_fast(C, s, sf, num_iterations, &cond, cnt);
    cond_set = true;
  }
  const float fcx = (float)f[DICEGPU_F_COORD_X], fcy = (float)f[DICEGPU_F_COORD_Y];
  float nu, nv, nt;
  sf.map_to_u_v_theta(fcx, fcy, nu, nv, nt);
  bool jump_pass = true;
  if (std::abs(nu - prev_u) > P.disp_jump_tol || std::abs(nv - prev_v) > P.disp_jump_tol ||
      std::abs(nt - prev_t) > P.theta_jump_tol)
    jump_pass = false;
  if (corr_status != DICEGPU_CORRELATION_SUCCESSFUL || !jump_pass) {
    bool second_failed = false;
    if (opt == DICEGPU_SIMPLEX || opt == DICEGPU_GRADIENT_BASED || force_simplex) {
      second_failed = true;
    } else if (opt == DICEGPU_GRADIENT_BASED_THEN_SIMPLEX) {
      init_status = initial_guess(f, nf, sf);
      corr_status = compute_update_robust(C, s, sf, num_iterations, cnt);
      if (corr_status != DICEGPU_CORRELATION_SUCCESSFUL) second_failed = true;
    } else if (opt == DICEGPU_SIMPLEX_THEN_GRADIENT_BASED) {
      init_status = initial_guess(f, nf, sf);
      corr_status = compute_update_fast(C, s, sf, num_iterations, &cond, cnt);
      cond_set = true;
      if (corr_status != DICEGPU_CORRELATION_SUCCESSFUL) second_failed = true;
    }
    if (second_failed && corr_status != DICEGPU_CORRELATION_SUCCESSFUL) {
      if (cond_set) f[DICEGPU_F_CONDITION] = cond;
      record_failed_step(f, corr_status, num_iterations);
      return false;
    }
  }
  if (cond_set) f[DICEGPU_F_CONDITION] = cond;
  float noise = 0.0f;
  const float sigma = objective_sigma(C, s, sf, noise);
  if (sigma < 0.0f) {
    record_failed_step(f, DICEGPU_FRAME_FAILED_DUE_TO_NEGATIVE_SIGMA, num_iterations);
    return false;
  }
  const float gamma = objective_gamma(C, s, sf, cnt);
  const float beta = P.output_beta ? objective_beta(C, s, sf) : 0.0f;
  if ((P.final_gamma_threshold != -1.0 && gamma > P.final_gamma_threshold) || gamma < 0.0f) {
    record_failed_step(f, DICEGPU_FRAME_FAILED_DUE_TO_HIGH_GAMMA, num_iterations);
    return false;
  }
  sf.map_to_u_v_theta(fcx, fcy, nu, nv, nt);
  if (std::abs(nu - prev_u) > P.disp_jump_tol || std::abs(nv - prev_v) > P.disp_jump_tol ||
      std::abs(nt - prev_t) > P.theta_jump_tol) {
    record_failed_step(f, DICEGPU_JUMP_TOLERANCE_EXCEEDED, num_iterations);
    return false;
  }
  const float contrast = s.contrast_std_dev();
  const int active_pixels = s.num_active();
  // record_step (DICe_Schema.cpp:1986-2009)
  sf.to_fields(f, (float)s.cx, (float)s.cy);
  f[DICEGPU_F_SIGMA] = sigma;
  f[DICEGPU_F_MATCH] = 0.0;
  f[DICEGPU_F_GAMMA] = gamma;
  f[DICEGPU_F_BETA] = beta;
  f[DICEGPU_F_NOISE] = noise;
  f[DICEGPU_F_CONTRAST] = contrast;
  f[DICEGPU_F_ACTIVE_PIXELS] = active_pixels;
  f[DICEGPU_F_STATUS] = init_status;
  f[DICEGPU_F_ITERATIONS] = num_iterations;
  return true;
}

}  // namespace oracle

using namespace oracle;

extern "C" int oracle_default_params(dicegpu_params* p) {
  if (!p) return DICEGPU_ERR_ARG;
  std::memset(p, 0, sizeof(*p));
  p->shape_function = DICEGPU_AFFINE_SF;
  p->enable_translation = 1;
  p->interpolation = DICEGPU_KEYS_FOURTH;
  p->optimization = DICEGPU_GRADIENT_BASED_THEN_SIMPLEX;
  p->gradient_method = DICEGPU_FINITE_DIFFERENCE;
  p->max_solver_iterations_fast = 25;
  p->max_solver_iterations_robust = 1000;
  p->fast_solver_tolerance = 1.0e-4;
  p->robust_solver_tolerance = 1.0e-6;
  p->skip_solve_gamma_threshold = 1.0e-10;
  p->robust_delta_disp = 1.0;
  p->robust_delta_theta = 0.1;
  p->disp_jump_tol = 10000.0;
  p->theta_jump_tol = 100.0;
  p->levenberg_marquardt_regularization_factor = -1.0;
  p->momentum_factor = 0.0;
  p->initial_gamma_threshold = -1.0;
  p->final_gamma_threshold = -1.0;
  p->use_def_gradients = 1;
  p->subset_size = 21;
  p->gauss_filter_images = 0;
  p->gauss_filter_mask_size = 7;
  p->correlation_routine = DICEGPU_GENERIC_ROUTINE;
  p->obstruction_skin_factor = 1.0;
  return 0;
}

extern "C" int oracle_gauss_filter(int w, int h, const float* in, float* out, int mask_size) {
  if (!in || !out || w < 1 || h < 1) return DICEGPU_ERR_ARG;
  return gauss_filter(w, h, mask_size, in, out) ? 0 : DICEGPU_ERR_ARG;
}

extern "C" int oracle_map(const dicegpu_params* params, const double* fields, int n, const float* xy,
                          float cx, float cy, float* out_xy) {
  if (!params || !fields || !xy || !out_xy || n < 0) return DICEGPU_ERR_ARG;
  ShapeFn sf;
  sf.init(*params);
  sf.from_fields(fields);
  for (int i = 0; i < n; ++i) sf.map(xy[2 * i], xy[2 * i + 1], cx, cy, out_xy[2 * i], out_xy[2 * i + 1]);
  return 0;
}

extern "C" int oracle_gradients(int w, int h, const float* img, int method, float* gx, float* gy) {
  if (w < 3 || h < 3 || !img || !gx || !gy) return DICEGPU_ERR_ARG;
  compute_gradients(w, h, img, method, gx, gy);
  return 0;
}

extern "C" int oracle_interpolate(int method, int w, int h, const float* img, const float* gx,
                                  const float* gy, int n, const float* xy, float* out_i,
                                  float* out_gx, float* out_gy) {
  if (!img || !xy || !out_i || n < 0) return DICEGPU_ERR_ARG;
  Image im;
  im.w = w; im.h = h; im.I = img; im.gx = gx; im.gy = gy;
  im.has_gradients = gx && gy && out_gx && out_gy;
  for (int k = 0; k < n; ++k) {
    float iv = 0.0f, a = 0.0f, b = 0.0f;
    interpolate(im, method, iv, a, b, im.has_gradients, xy[2 * k], xy[2 * k + 1]);
    out_i[k] = iv;
    if (im.has_gradients) { out_gx[k] = a; out_gy[k] = b; }
  }
  return 0;
}

namespace {
// buffers a frame's images and gradients live in
struct FrameStore {
  std::vector<float> fref, fdef, rgx, rgy, dgx, dgy;
};

struct FrameJob {
  std::shared_ptr<FrameStore> store;
  Ctx C;
  int n;
  double* fields;
  const int32_t *offsets, *px, *py;
  const uint8_t* force_simplex;
  bool first_frame;
  int32_t* gn_out;
  int32_t* sx_out;
  double* unc;
  const std::vector<PixelSet>* obst = nullptr;   // per subset
  const PixelSet* blocked = nullptr;             // the subset being run (tracking order)
  uint8_t* pix_flag = nullptr;                   // subset evolution state per list pixel
  float* pix_f = nullptr;
  bool evolve = false;                           // turn on visible inactive pixels after success
  const int32_t* neighbors = nullptr;            // neighbour initialization this frame
};

void run_range(const FrameJob& J, int b, int e) {
  Subset s;
  for (int i = b; i < e; ++i) {
    double* f = J.fields + (long)i * DICEGPU_FIELD_STRIDE;
    const int cx = (int)f[DICEGPU_F_COORD_X], cy = (int)f[DICEGPU_F_COORD_Y];
    if (J.offsets) s.init_list(cx, cy, J.px + J.offsets[i], J.py + J.offsets[i],
                               J.offsets[i + 1] - J.offsets[i]);
    else s.init_square(cx, cy, J.C.P.subset_size);
    s.flag = J.pix_flag ? J.pix_flag + J.offsets[i] : nullptr;
    s.fstore = J.pix_f ? J.pix_f + J.offsets[i] : nullptr;
    s.init_ref(J.C.ref);
    s.obstructed = J.obst ? &(*J.obst)[i] : nullptr;
    s.blocked = J.blocked;
    Counters cnt;
    if (J.unc) {
      cnt.unc = J.unc + (long)i * DICEGPU_UNCERTAINTY_STRIDE;
      cnt.ucx = (float)f[DICEGPU_F_COORD_X];
      cnt.ucy = (float)f[DICEGPU_F_COORD_Y];
    }
    // neighbour initialization: subsets run in index order, so a lower
    // neighbour's row holds this frame's solution, a higher one's the
    // previous frame's
    const double* nf = nullptr;
    if (J.neighbors) {
      const int j = J.neighbors[i];
      if (j >= 0 && j < J.n && j != i) nf = J.fields + (long)j * DICEGPU_FIELD_STRIDE;
    }
    const bool ok = correlate_subset(J.C, s, f, J.first_frame, J.force_simplex ? J.force_simplex[i] : 0u, &cnt, nf);
    // Subset::turn_on_previously_obstructed_pixels (DICe_Subset.cpp:506-520)
    // with the deformed state of the last evaluation
    if (ok && J.evolve && s.flag)
      for (int k = 0; k < s.npix; ++k)
        if (!s.active[k] && !s.deact[k]) {
          s.fstore[k] = s.def[k];
          s.flag[k] = 2;
        }
    if (J.gn_out) J.gn_out[i] = cnt.gn_iters;
    if (J.sx_out) J.sx_out[i] = cnt.simplex_evals;
  }
}
}  // namespace

// images, gradients and parameters of a frame (the images' optional Gaussian
// pre-filter comes before their gradients)
static int prepare_frame(const dicegpu_params* params, int w, int h, const float* ref, const float* def,
                         FrameJob& J) {
  if (!params || !ref || !def || w < 16 || h < 16) return DICEGPU_ERR_ARG;
  J.store.reset(new FrameStore());
  FrameStore& S = *J.store;
  if (params->gauss_filter_images) {
    S.fref.resize((long)w * h);
    S.fdef.resize((long)w * h);
    if (!gauss_filter(w, h, params->gauss_filter_mask_size, ref, S.fref.data()) ||
        !gauss_filter(w, h, params->gauss_filter_mask_size, def, S.fdef.data()))
      return DICEGPU_ERR_ARG;
    ref = S.fref.data();
    def = S.fdef.data();
  }
  J.C.P = *params;
  // gradients as Schema::set_ref_image / set_def_image compute them
  S.rgx.resize((long)w * h);
  S.rgy.resize((long)w * h);
  compute_gradients(w, h, ref, params->gradient_method, S.rgx.data(), S.rgy.data());
  J.C.ref.w = w; J.C.ref.h = h; J.C.ref.I = ref;
  J.C.ref.gx = S.rgx.data(); J.C.ref.gy = S.rgy.data(); J.C.ref.has_gradients = true;
  J.C.def.w = w; J.C.def.h = h; J.C.def.I = def;
  if (params->use_def_gradients) {
    S.dgx.resize((long)w * h); S.dgy.resize((long)w * h);
    compute_gradients(w, h, def, params->gradient_method, S.dgx.data(), S.dgy.data());
    J.C.def.gx = S.dgx.data(); J.C.def.gy = S.dgy.data(); J.C.def.has_gradients = true;
  }
  return 0;
}

static void run_parallel(const FrameJob& J, int nthreads) {
  const int n = J.n;
  if (nthreads <= 1 || n < 2 || J.neighbors) {   // neighbour chains run in index order
    run_range(J, 0, n);
    return;
  }
  if (nthreads > n) nthreads = n;
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) {
    const int b = (int)((long)n * t / nthreads), e = (int)((long)n * (t + 1) / nthreads);
    th.emplace_back(run_range, std::cref(J), b, e);
  }
  for (auto& x : th) x.join();
}

extern "C" int oracle_execute_frame(const dicegpu_params* params, int w, int h, const float* ref,
                                    const float* def, int n, double* fields,
                                    const int32_t* offsets, const int32_t* px,
                                    const int32_t* py, const uint8_t* force_simplex,
                                    int first_frame, int nthreads, int32_t* gn_iters_out,
                                    int32_t* simplex_evals_out, double* uncertainty, const int32_t* neighbors) {
  if (!fields || n < 0) return DICEGPU_ERR_ARG;
  FrameJob J;
  const int rc = prepare_frame(params, w, h, ref, def, J);
  if (rc) return rc;
  const int im = params->initialization_method;
  if (im != DICEGPU_USE_FIELD_VALUES && im != DICEGPU_USE_NEIGHBOR_VALUES &&
      im != DICEGPU_USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY)
    return DICEGPU_ERR_UNSUPPORTED;
  if (neighbors && (im == DICEGPU_USE_NEIGHBOR_VALUES || (im == DICEGPU_USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY && first_frame)))
    J.neighbors = neighbors;
  J.n = n; J.fields = fields; J.offsets = offsets; J.px = px; J.py = py;
  J.force_simplex = force_simplex; J.first_frame = first_frame != 0;
  J.gn_out = gn_iters_out; J.sx_out = simplex_evals_out; J.unc = uncertainty;
  run_parallel(J, nthreads);
  return 0;
}

// The Gauss-Newton system of Objective_ZNSSD::computeUpdateFast
// (DICe_Objective.cpp:523-546) assembled once, for a fresh square subset at
// the parameters of each field row: H (n x N x N) and q (n x N), compact
// parameter order.  No solve.
extern "C" int oracle_gn_system(const dicegpu_params* params, int w, int h, const float* ref,
                                const float* def, int n, const double* fields, double* H_out,
                                double* q_out) {
  if (!params || !ref || !def || !fields || !H_out || !q_out) return DICEGPU_ERR_ARG;
  Ctx C;
  C.P = *params;
  std::vector<float> rgx((long)w * h), rgy((long)w * h), dgx, dgy;
  compute_gradients(w, h, ref, params->gradient_method, rgx.data(), rgy.data());
  C.ref.w = w; C.ref.h = h; C.ref.I = ref; C.ref.gx = rgx.data(); C.ref.gy = rgy.data();
  C.ref.has_gradients = true;
  C.def.w = w; C.def.h = h; C.def.I = def;
  if (params->use_def_gradients) {
    dgx.resize((long)w * h); dgy.resize((long)w * h);
    compute_gradients(w, h, def, params->gradient_method, dgx.data(), dgy.data());
    C.def.gx = dgx.data(); C.def.gy = dgy.data(); C.def.has_gradients = true;
  }
  const bool use_ref_grads = !C.def.has_gradients;
  Subset s;
  for (int i = 0; i < n; ++i) {
    const double* f = fields + (long)i * DICEGPU_FIELD_STRIDE;
    s.init_square((int)f[DICEGPU_F_COORD_X], (int)f[DICEGPU_F_COORD_Y], params->subset_size);
    s.init_ref(C.ref);
    ShapeFn sf;
    sf.init(C.P);
    sf.from_fields(f);
    const int N = sf.N;
    double* H = H_out + (long)i * N * N;
    double* q = q_out + (long)i * N;
    for (int k = 0; k < N * N; ++k) H[k] = 0.0;
    for (int k = 0; k < N; ++k) q[k] = 0.0;
    const float meanF = s.mean(false);
    s.init_def(C.def, sf, C.P.interpolation);
    const float meanG = s.mean(true);
    const float fcx = (float)s.cx, fcy = (float)s.cy;
    float r[12];
    for (int idx = 0; idx < s.npix; ++idx) {
      if (s.deact[idx] || !s.active[idx]) continue;
      const float GmF = (s.def[idx] - meanG) - (s.ref[idx] - meanF);
      for (int k = 0; k < N; ++k) r[k] = 0.0f;
      sf.residuals((float)s.x[idx], (float)s.y[idx], fcx, fcy, s.gx[idx], s.gy[idx], r,
                   use_ref_grads);
      for (int a = 0; a < N; ++a) {
        q[a] += GmF * r[a];
        for (int b = 0; b < N; ++b) H[a * N + b] += r[a] * r[b];
      }
    }
  }
  return 0;
}

// Pixel ownership of the conformal-subset shapes without deformation
// (Circle / Rectangle / Polygon::get_owned_pixels, DICe_Shape.cpp:136-219,
// 259-279, 322-420) and of excluded shapes (deactivate_pixels, :104-134,
// 233-256, 298-320).  kind 0 circle (cx, cy, radius), 1 rectangle (cx, cy,
// width, height), 2 polygon (vertices).
namespace {
// angle_2d (DICe_Shape.cpp:87-102): float atan2 of float arguments, the
// wrap against the double constants, result stored as float.  The float
// atan2 is taken correctly rounded (the double atan2 rounded to float): a
// pixel lying exactly on a polygon edge sees that edge's term at +-pi, and
// which side of pi it rounds to follows the last bit of atan2f, which
// differs between math libraries (glibc 2.39's atan2f is 1 ulp off on ~16 %
// of small integer vectors and flips ~2.5 % of on-edge pixels).  Correct
// rounding fixes that choice everywhere and reproduces the reference's
// conformal-subset image; off the edges no pixel depends on it.
static float angle_2d(float x1, float y1, float x2, float y2) {
  float t1 = (float)std::atan2((double)y1, (double)x1), t2 = (float)std::atan2((double)y2, (double)x2);
  float d = t2 - t1;
  while (d > 3.14159265358979323846) d -= 6.28318530717958647692;
  while (d < -3.14159265358979323846) d += 6.28318530717958647692;
  return d;
}
// the winding-angle test over a closed vertex loop (vertex nv is vertex 0)
static bool polygon_has(const int32_t* vx, const int32_t* vy, int nv, int x, int y) {
  float angle = 0.0f;
  for (int i = 0; i < nv; ++i) {
    const int j = (i + 1 == nv) ? 0 : i + 1;
    const float dx1 = (float)(vx[i] - x), dy1 = (float)(vy[i] - y);
    const float dx2 = (float)(vx[j] - x), dy2 = (float)(vy[j] - y);
    angle += angle_2d(dx1, dy1, dx2, dy2);
  }
  return std::abs(angle) >= 3.14159265358979323846;
}
// get_owned_pixels' test (excluded = false) or deactivate_pixels' (true):
// they differ only in how the circle adds the squares
static bool shape_has(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, int x, int y,
                      bool excluded) {
  if (s.kind == 0) {
    const int lim = (int)s.radius + 1;   // outside; keeps the squares inside int
    if (std::abs(x - s.cx) > lim || std::abs(y - s.cy) > lim) return false;
    const float r2 = s.radius * s.radius;
    const int ix = (x - s.cx) * (x - s.cx), iy = (y - s.cy) * (y - s.cy);
    if (excluded) return (float)(ix + iy) <= r2;
    return (float)ix + (float)iy <= r2;
  }
  if (s.kind == 1) {
    const int ox = s.cx - s.width / 2, oy = s.cy - s.height / 2;
    return x >= ox && x < ox + s.width && y >= oy && y < oy + s.height;
  }
  return polygon_has(vx + s.vertex_offset, vy + s.vertex_offset, s.vertex_count, x, y);
}
static void shape_box(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, int& x0, int& x1,
                      int& y0, int& y1) {
  if (s.kind == 0) {
    x0 = (int)((float)s.cx - s.radius - 1.0f); x1 = (int)((float)s.cx + s.radius + 1.0f);
    y0 = (int)((float)s.cy - s.radius - 1.0f); y1 = (int)((float)s.cy + s.radius + 1.0f);
  } else if (s.kind == 1) {
    x0 = s.cx - s.width / 2; x1 = x0 + s.width - 1;
    y0 = s.cy - s.height / 2; y1 = y0 + s.height - 1;
  } else {
    x0 = x1 = vx[s.vertex_offset];
    y0 = y1 = vy[s.vertex_offset];
    for (int i = 1; i < s.vertex_count; ++i) {
      x0 = std::min(x0, vx[s.vertex_offset + i]); x1 = std::max(x1, vx[s.vertex_offset + i]);
      y0 = std::min(y0, vy[s.vertex_offset + i]); y1 = std::max(y1, vy[s.vertex_offset + i]);
    }
  }
}
// owned pixels of one undeformed shape
static void owned_pixels(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, PixelSet& out) {
  int x0, x1, y0, y1;
  shape_box(s, vx, vy, x0, x1, y0, y1);
  for (int y = y0; y <= y1; ++y)
    for (int x = x0; x <= x1; ++x)
      if (shape_has(s, vx, vy, x, y, false)) out.insert(std::make_pair(y, x));
}
// Polygon / Rectangle::get_owned_pixels with a shape function
// (DICe_Shape.cpp:136-219, 322-396): the vertices mapped and rounded, then
// stretched by skin about their integer centroid, then the winding test.  A
// rectangle is the loop (o), (o + w, o), (o + w, o + h), (o, o + h).
static void deformed_pixels(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy,
                            const ShapeFn& sf, int cx, int cy, float skin, PixelSet& out) {
  std::vector<int32_t> X, Y;
  if (s.kind == 1) {
    const int ox = s.cx - s.width / 2, oy = s.cy - s.height / 2;
    X = {ox, ox + s.width, ox + s.width, ox};
    Y = {oy, oy, oy + s.height, oy + s.height};
  } else {
    X.assign(vx + s.vertex_offset, vx + s.vertex_offset + s.vertex_count);
    Y.assign(vy + s.vertex_offset, vy + s.vertex_offset + s.vertex_count);
  }
  const int nv = (int)X.size();
  for (int i = 0; i < nv; ++i) {
    float mx, my;
    sf.map((float)X[i], (float)Y[i], (float)cx, (float)cy, mx, my);
    int nx = (int)mx;
    if (mx - (float)(int)mx >= 0.5) nx++;
    int ny = (int)my;
    if (my - (float)(int)my >= 0.5) ny++;
    X[i] = nx;
    Y[i] = ny;
  }
  // integer centroid, divided as a double and truncated
  int sx = 0, sy = 0;
  for (int i = 0; i < nv; ++i) { sx += X[i]; sy += Y[i]; }
  const int ccx = (int)((double)sx / (double)nv), ccy = (int)((double)sy / (double)nv);
  int x0 = 0, x1 = 0, y0 = 0, y1 = 0;
  for (int i = 0; i < nv; ++i) {
    const float fx = skin * (float)(X[i] - ccx);
    const float fy = skin * (float)(Y[i] - ccy);
    X[i] = (int)(fx + (float)ccx);
    Y[i] = (int)(fy + (float)ccy);
    if (i == 0) { x0 = x1 = X[i]; y0 = y1 = Y[i]; }
    else {
      x0 = std::min(x0, X[i]); x1 = std::max(x1, X[i]);
      y0 = std::min(y0, Y[i]); y1 = std::max(y1, Y[i]);
    }
  }
  for (int y = y0; y <= y1; ++y)
    for (int x = x0; x <= x1; ++x)
      if (polygon_has(X.data(), Y.data(), nv, x, y)) out.insert(std::make_pair(y, x));
}

// one subset's pixel list: the union of its boundary shapes in (y, x) order
// without the excluded pixels (tested at the clamped coordinates), or the
// square of `square_size` about its centroid when it has no boundary shape.
// With flags, the excluded pixels stay in the list with flag 0 (inactive),
// the others get flag 1.
static void subset_pixels(const std::vector<int>& mine, const dicegpu_shape* shapes, const int32_t* vx,
                          const int32_t* vy, int cx, int cy, int square_size, std::vector<int32_t>& px,
                          std::vector<int32_t>& py, std::vector<uint8_t>* flags = nullptr) {
  px.clear();
  py.clear();
  if (flags) flags->clear();
  int x0 = 0, x1 = -1, y0 = 0, y1 = -1;
  bool any = false;
  for (int k : mine) {
    if (shapes[k].role != DICEGPU_ROLE_BOUNDARY) continue;
    int a, b, c, d;
    shape_box(shapes[k], vx, vy, a, b, c, d);
    if (!any) { x0 = a; x1 = b; y0 = c; y1 = d; any = true; }
    else { x0 = std::min(x0, a); x1 = std::max(x1, b); y0 = std::min(y0, c); y1 = std::max(y1, d); }
  }
  if (!any) {
    if (square_size < 1) return;
    const int hw = square_size / 2;
    for (int y = cy - hw; y <= cy + hw; ++y)
      for (int x = cx - hw; x <= cx + hw; ++x) {
        px.push_back(x < 0 ? 0 : x);
        py.push_back(y < 0 ? 0 : y);
        if (flags) flags->push_back(1);
      }
    return;
  }
  for (int y = y0; y <= y1; ++y)
    for (int x = x0; x <= x1; ++x) {
      bool in = false, out = false;
      const int ex = x < 0 ? 0 : x, ey = y < 0 ? 0 : y;
      for (int k : mine) {
        if (shapes[k].role == DICEGPU_ROLE_BOUNDARY) in = in || shape_has(shapes[k], vx, vy, x, y, false);
        else if (shapes[k].role == DICEGPU_ROLE_EXCLUDED) out = out || shape_has(shapes[k], vx, vy, ex, ey, true);
      }
      if (in && (!out || flags)) {
        px.push_back(ex);
        py.push_back(ey);
        if (flags) flags->push_back(out ? 0 : 1);
      }
    }
}

static bool group_shapes(int n, int n_shapes, const dicegpu_shape* shapes, std::vector<std::vector<int>>& by) {
  by.assign(n, {});
  for (int k = 0; k < n_shapes; ++k) {
    if (shapes[k].subset < 0 || shapes[k].subset >= n) return false;
    by[shapes[k].subset].push_back(k);
  }
  return true;
}
}  // namespace

// Pixel lists of n subsets from their shapes (Subset(cx, cy,
// Conformal_Area_Def), DICe_Subset.cpp:115-168; negative coordinates clamped
// to 0).  Subsets without boundary shapes are squares of square_size about
// the field rows' coordinates (fields may be NULL when every subset has
// boundary shapes).  With px == NULL only offsets[n+1] is filled.
extern "C" int oracle_rasterize(int n, int n_shapes, const dicegpu_shape* shapes, const int32_t* vx,
                                const int32_t* vy, const double* fields, int square_size,
                                int32_t* offsets, int32_t* px, int32_t* py) {
  if (n < 0 || n_shapes < 0 || !offsets || (n_shapes && !shapes)) return DICEGPU_ERR_ARG;
  std::vector<std::vector<int>> by;
  if (!group_shapes(n, n_shapes, shapes, by)) return DICEGPU_ERR_ARG;
  offsets[0] = 0;
  std::vector<int32_t> lx, ly;
  for (int i = 0; i < n; ++i) {
    const int cx = fields ? (int)fields[(long)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X] : 0;
    const int cy = fields ? (int)fields[(long)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y] : 0;
    subset_pixels(by[i], shapes, vx, vy, cx, cy, fields ? square_size : 0, lx, ly);
    if (px)
      for (size_t k = 0; k < lx.size(); ++k) { px[offsets[i] + k] = lx[k]; py[offsets[i] + k] = ly[k]; }
    offsets[i + 1] = offsets[i] + (int32_t)lx.size();
  }
  return 0;
}

// Schema::execute_correlation for subsets defined by shapes, with
// obstructions and blocking subsets (see dicegpu_set_subset_shapes and
// dicegpu_set_blocking).  The generic routine runs the subsets in threads;
// the tracking routine with blocking runs them in index order, each blocked
// subset's blocked pixels taken from its blockers' fields as they stand
// (check_for_blocking_subsets, DICe_Schema.cpp:4529-4557).  Blocked and
// blocking subsets take the simplex unless params.override_force_simplex
// (DICe_Schema.cpp:2160-2185).
extern "C" int oracle_execute_frame_shapes(const dicegpu_params* params, int w, int h, const float* ref,
                                           const float* def, int n, double* fields, int n_shapes,
                                           const dicegpu_shape* shapes, const int32_t* vx,
                                           const int32_t* vy, const int32_t* block_offsets,
                                           const int32_t* block_ids, const uint8_t* force_simplex,
                                           int first_frame, int nthreads, uint8_t* pix_flag, float* pix_f,
                                           int frame_index) {
  if (!params || !fields || n < 1) return DICEGPU_ERR_ARG;
  std::vector<std::vector<int>> by;
  if (!group_shapes(n, n_shapes, shapes, by)) return DICEGPU_ERR_ARG;
  // the tracking routine's objectives persist across frames and carry the
  // evolved subsets (DICe_Schema.cpp:1729-1748); the generic routine's are
  // rebuilt every frame (:1708-1724)
  const bool evolution = params->use_subset_evolution != 0 && params->correlation_routine == DICEGPU_TRACKING_ROUTINE;
  // pixel lists and obstruction sets
  std::vector<int32_t> offsets(n + 1, 0), px, py, lx, ly;
  std::vector<uint8_t> flags, lf;
  std::vector<PixelSet> obst(n);
  std::vector<char> conformal(n, 0);
  for (int i = 0; i < n; ++i) {
    const double* f = fields + (long)i * DICEGPU_FIELD_STRIDE;
    subset_pixels(by[i], shapes, vx, vy, (int)f[DICEGPU_F_COORD_X], (int)f[DICEGPU_F_COORD_Y],
                  params->subset_size, lx, ly, evolution ? &lf : nullptr);
    px.insert(px.end(), lx.begin(), lx.end());
    py.insert(py.end(), ly.begin(), ly.end());
    flags.insert(flags.end(), lf.begin(), lf.end());
    offsets[i + 1] = offsets[i] + (int32_t)lx.size();
    for (int k : by[i]) {
      if (shapes[k].role == DICEGPU_ROLE_OBSTRUCTED) owned_pixels(shapes[k], vx, vy, obst[i]);
      if (shapes[k].role == DICEGPU_ROLE_BOUNDARY) conformal[i] = 1;
    }
  }
  // forced simplex: the caller's flags, blocked and blocking subsets
  std::vector<uint8_t> force(n, 0);
  for (int i = 0; i < n; ++i) force[i] = force_simplex ? force_simplex[i] : 0;
  bool any_block = false;
  if (block_offsets) {
    for (int i = 0; i < n; ++i)
      for (int k = block_offsets[i]; k < block_offsets[i + 1]; ++k) {
        if (block_ids[k] < 0 || block_ids[k] >= n) return DICEGPU_ERR_ARG;
        any_block = true;
        if (!params->override_force_simplex) { force[i] |= 1; force[block_ids[k]] |= 1; }
      }
  }
  FrameJob J;
  const int rc = prepare_frame(params, w, h, ref, def, J);
  if (rc) return rc;
  J.n = n; J.fields = fields; J.offsets = offsets.data(); J.px = px.data(); J.py = py.data();
  J.force_simplex = force.data(); J.first_frame = first_frame != 0;
  J.gn_out = nullptr; J.sx_out = nullptr; J.unc = nullptr;
  J.obst = &obst;
  // subset evolution: the caller's state (initialised at the sequence's first frame)
  std::vector<float> fstore;
  if (evolution) {
    if (pix_flag && pix_f) {
      if (frame_index == 0) {
        std::copy(flags.begin(), flags.end(), pix_flag);
        std::fill(pix_f, pix_f + flags.size(), 0.0f);
      }
      J.pix_flag = pix_flag;
      J.pix_f = pix_f;
    } else {
      fstore.assign(flags.size(), 0.0f);
      J.pix_flag = flags.data();
      J.pix_f = fstore.data();
    }
    // turned on from the third frame (frame_id_ > first_frame_id_ + frame_skip_)
    J.evolve = frame_index >= 2;
  }
  const bool tracking = params->correlation_routine == DICEGPU_TRACKING_ROUTINE && any_block;
  if (!tracking) {
    run_parallel(J, nthreads);
    return 0;
  }
  ShapeFn sf;
  sf.init(J.C.P);
  for (int i = 0; i < n; ++i) {
    PixelSet blocked;
    for (int k = block_offsets[i]; k < block_offsets[i + 1]; ++k) {
      const int j = block_ids[k];
      if (!conformal[j]) continue;   // deformed_shapes of a square subset is empty
      const double* fj = fields + (long)j * DICEGPU_FIELD_STRIDE;
      ShapeFn sj = sf;
      sj.from_fields(fj);
      for (int m : by[j]) {
        if (shapes[m].role != DICEGPU_ROLE_BOUNDARY) continue;
        if (shapes[m].kind == 0) return DICEGPU_ERR_UNSUPPORTED;   // circle deformation throws
        deformed_pixels(shapes[m], vx, vy, sj, (int)fj[DICEGPU_F_COORD_X], (int)fj[DICEGPU_F_COORD_Y],
                        (float)params->obstruction_skin_factor, blocked);
      }
    }
    J.blocked = &blocked;
    run_range(J, i, i + 1);
    J.blocked = nullptr;
  }
  return 0;
}

// VSG_Strain_Post_Processor::execute (DICe_PostProcessor.cpp:931-1130) with
// its neighbourhoods (Post_Processor::initialize_neighborhood, :140-236,
// radius search): for every point the points within window/2 (float
// squared distance < r^2 + 1e-5, the kd-tree's test), sorted by distance;
// the neighbours with sigma >= 0 fit u and v by a plane [1, dx, dy] in
// double; fewer than 3, an invalid point, or a condition estimate below
// 1e-12 give zeros and MATCH = -1.  The condition number is computed
// exactly here (||A||_1 ||A^-1||_1) where the reference estimates it with
// GECON; the test differs only for nearly collinear neighbourhoods.
// Field values are the reference's floats.  out: n x 7 (strain xx, yy, xy,
// du/dx, du/dy, dv/dx, dv/dy), failed: n flags.
namespace {
// LU with partial pivoting and the inverse of a 3 x 3 (GETRF / GETRI);
// false when a pivot is exactly 0
static bool inverse3(const double A_in[3][3], double inv[3][3]) {
  double A[3][3];
  int piv[3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) A[i][j] = A_in[i][j];
  for (int k = 0; k < 3; ++k) {
    int p = k;
    for (int i = k + 1; i < 3; ++i)
      if (std::fabs(A[i][k]) > std::fabs(A[p][k])) p = i;
    piv[k] = p;
    if (A[p][k] == 0.0) return false;
    if (p != k)
      for (int j = 0; j < 3; ++j) std::swap(A[k][j], A[p][j]);
    for (int i = k + 1; i < 3; ++i) {
      A[i][k] /= A[k][k];
      for (int j = k + 1; j < 3; ++j) A[i][j] -= A[i][k] * A[k][j];
    }
  }
  // solve A X = I column by column (the row interchanges applied to I)
  for (int c = 0; c < 3; ++c) {
    double b[3] = {0.0, 0.0, 0.0};
    b[c] = 1.0;
    for (int k = 0; k < 3; ++k) std::swap(b[k], b[piv[k]]);
    for (int i = 1; i < 3; ++i)
      for (int j = 0; j < i; ++j) b[i] -= A[i][j] * b[j];
    for (int i = 2; i >= 0; --i) {
      for (int j = i + 1; j < 3; ++j) b[i] -= A[i][j] * b[j];
      b[i] /= A[i][i];
    }
    for (int i = 0; i < 3; ++i) inv[i][c] = b[i];
  }
  return true;
}
static double norm1(const double M[3][3]) {
  double a = 0.0;
  for (int j = 0; j < 3; ++j) {
    double c = 0.0;
    for (int i = 0; i < 3; ++i) c += std::fabs(M[i][j]);
    a = std::max(a, c);
  }
  return a;
}
}  // namespace

// window > 0: the neighbours within window / 2 (the kd-tree radius search,
// DICe_PostProcessor.cpp:207-231); window < 0: the -window nearest points,
// valid or not (knnSearch, :185-205), by float squared distance, ties by
// index (the kd-tree breaks ties by its traversal order).
extern "C" int oracle_vsg_strain(int n, const double* fields, int window, double* out, int32_t* failed) {
  if (n < 1 || !fields || !out || !failed || window == 0) return DICEGPU_ERR_ARG;
  if (window < 0 && -(long)window > n) return DICEGPU_ERR_ARG;
  const int knn = window < 0 ? -window : 0;
  const float rad = (float)((float)(window < 0 ? 1 : window) / 2.0);
  const float r2 = rad * rad + 1.0e-5f;
  std::vector<float> px(n), py(n), u(n), v(n), sg(n);
  for (int i = 0; i < n; ++i) {
    const double* f = fields + (long)i * DICEGPU_FIELD_STRIDE;
    px[i] = (float)f[DICEGPU_F_COORD_X];
    py[i] = (float)f[DICEGPU_F_COORD_Y];
    u[i] = (float)f[DICEGPU_F_DISP_X];
    v[i] = (float)f[DICEGPU_F_DISP_Y];
    sg[i] = (float)f[DICEGPU_F_SIGMA];
  }
  // candidates from a uniform grid of cell size >= the radius + 1 (the
  // kd-tree's role: which points are tested, not how)
  const float cell = std::ceil(std::sqrt(r2)) + 1.0f;
  float x0 = px[0], y0 = py[0], x1 = px[0], y1 = py[0];
  for (int i = 1; i < n; ++i) {
    x0 = std::min(x0, px[i]); x1 = std::max(x1, px[i]);
    y0 = std::min(y0, py[i]); y1 = std::max(y1, py[i]);
  }
  const long ncx = (long)std::floor((x1 - x0) / cell) + 1, ncy = (long)std::floor((y1 - y0) / cell) + 1;
  std::map<long, std::vector<int>> cells;
  auto cell_of = [&](int i) {
    return (long)std::floor((py[i] - y0) / cell) * ncx + (long)std::floor((px[i] - x0) / cell);
  };
  if (knn == 0)
    for (int i = 0; i < n; ++i) cells[cell_of(i)].push_back(i);
  std::vector<std::pair<float, int>> nb;
  for (int i = 0; i < n; ++i) {
    nb.clear();
    if (knn > 0) {
      // every point, the knn smallest
      for (int j = 0; j < n; ++j) {
        const float dx = px[i] - px[j], dy = py[i] - py[j];
        nb.push_back(std::make_pair(dx * dx + dy * dy, j));
      }
      std::sort(nb.begin(), nb.end());
      nb.resize(knn);
    } else {
      const long gx = (long)std::floor((px[i] - x0) / cell), gy = (long)std::floor((py[i] - y0) / cell);
      for (long cy = std::max(gy - 1, 0L); cy <= std::min(gy + 1, ncy - 1); ++cy)
        for (long cx = std::max(gx - 1, 0L); cx <= std::min(gx + 1, ncx - 1); ++cx) {
          const auto it = cells.find(cy * ncx + cx);
          if (it == cells.end()) continue;
          for (int j : it->second) {
            const float dx = px[i] - px[j], dy = py[i] - py[j];
            const float d2 = dx * dx + dy * dy;
            if (d2 < r2) nb.push_back(std::make_pair(d2, j));
          }
        }
      // distance order, ties by index
      std::sort(nb.begin(), nb.end());
    }
    double* o = out + (long)i * 7;
    for (int k = 0; k < 7; ++k) o[k] = 0.0;
    failed[i] = 1;
    int valid = 0;
    for (const auto& q : nb) valid += sg[q.second] >= 0.0f;
    if (valid < 3 || nb.empty() || sg[nb[0].second] < 0.0f) continue;
    double XtX[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}}, Xu[3] = {0, 0, 0}, Xv[3] = {0, 0, 0};
    for (const auto& q : nb) {
      const int j = q.second;
      if (!(sg[j] >= 0.0f)) continue;
      const double row[3] = {1.0, (double)(px[j] - px[i]), (double)(py[j] - py[i])};
      for (int a = 0; a < 3; ++a) {
        for (int b = 0; b < 3; ++b) XtX[a][b] += row[a] * row[b];
        Xu[a] += row[a] * (double)u[j];
        Xv[a] += row[a] * (double)v[j];
      }
    }
    double inv[3][3];
    if (!inverse3(XtX, inv)) continue;
    const double rcond = 1.0 / (norm1(XtX) * norm1(inv));
    if (rcond < 1.0e-12) continue;
    double cx[3] = {0, 0, 0}, cy[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        cx[a] += inv[a][b] * Xu[b];
        cy[a] += inv[a][b] * Xv[b];
      }
    const double dudx = cx[1], dudy = cx[2], dvdx = cy[1], dvdy = cy[2];
    o[0] = (float)(0.5 * (2.0 * dudx + dudx * dudx + dvdx * dvdx));
    o[1] = (float)(0.5 * (2.0 * dvdy + dudy * dudy + dvdy * dvdy));
    o[2] = (float)(0.5 * (dudy + dvdx + dudx * dudy + dvdx * dvdy));
    o[3] = (float)dudx;
    o[4] = (float)dudy;
    o[5] = (float)dvdx;
    o[6] = (float)dvdy;
    failed[i] = 0;
  }
  return 0;
}

// One Objective entry point per subset on a fresh square subset at the
// parameters of its field row: op 0 computeUpdateFast (:430-657), op 1
// computeUpdateRobust (:369-388), op 2 sigma (:150-184) after the subset's
// deformed-state initialisation at those parameters.  Ops 0 and 1 write the
// shape-function fields (and CONDITION for op 0) back into `fields`.
extern "C" int oracle_objective(const dicegpu_params* params, int w, int h, const float* ref,
                                const float* def, int n, double* fields, int op, int32_t* iters_out,
                                int32_t* status_out, double* sigma_out, double* noise_out) {
  if (!params || !ref || !def || !fields || op < 0 || op > 2) return DICEGPU_ERR_ARG;
  std::vector<float> fref, fdef;
  if (params->gauss_filter_images) {
    fref.resize((long)w * h);
    fdef.resize((long)w * h);
    if (!gauss_filter(w, h, params->gauss_filter_mask_size, ref, fref.data()) ||
        !gauss_filter(w, h, params->gauss_filter_mask_size, def, fdef.data()))
      return DICEGPU_ERR_ARG;
    ref = fref.data();
    def = fdef.data();
  }
  Ctx C;
  C.P = *params;
  std::vector<float> rgx((long)w * h), rgy((long)w * h), dgx, dgy;
  compute_gradients(w, h, ref, params->gradient_method, rgx.data(), rgy.data());
  C.ref.w = w; C.ref.h = h; C.ref.I = ref; C.ref.gx = rgx.data(); C.ref.gy = rgy.data();
  C.ref.has_gradients = true;
  C.def.w = w; C.def.h = h; C.def.I = def;
  if (params->use_def_gradients) {
    dgx.resize((long)w * h); dgy.resize((long)w * h);
    compute_gradients(w, h, def, params->gradient_method, dgx.data(), dgy.data());
    C.def.gx = dgx.data(); C.def.gy = dgy.data(); C.def.has_gradients = true;
  }
  Subset s;
  for (int i = 0; i < n; ++i) {
    double* f = fields + (long)i * DICEGPU_FIELD_STRIDE;
    s.init_square((int)f[DICEGPU_F_COORD_X], (int)f[DICEGPU_F_COORD_Y], params->subset_size);
    s.init_ref(C.ref);
    ShapeFn sf;
    sf.init(C.P);
    sf.from_fields(f);
    const float fcx = (float)f[DICEGPU_F_COORD_X], fcy = (float)f[DICEGPU_F_COORD_Y];
    if (op == 2) {
      s.init_def(C.def, sf, C.P.interpolation);
      float noise = 0.0f;
      const float sg = objective_sigma(C, s, sf, noise);
      if (sigma_out) sigma_out[i] = sg;
      if (noise_out) noise_out[i] = noise;
      continue;
    }
    int num_iterations = -1, st;
    if (op == 0) {
      double cond = 0.0;
      st = compute_update_fast(C, s, sf, num_iterations, &cond, nullptr);
      f[DICEGPU_F_CONDITION] = cond;
    } else {
      st = compute_update_robust(C, s, sf, num_iterations, nullptr);
    }
    sf.to_fields(f, fcx, fcy);
    if (iters_out) iters_out[i] = num_iterations;
    if (status_out) status_out[i] = st;
  }
  return 0;
}

extern "C" int oracle_gamma(const dicegpu_params* params, int w, int h, const float* ref,
                            const float* def, int n, const double* fields, double* gamma_out) {
  if (!params || !ref || !def || !fields || !gamma_out) return DICEGPU_ERR_ARG;
  std::vector<float> fref, fdef;
  if (params->gauss_filter_images) {
    fref.resize((long)w * h);
    fdef.resize((long)w * h);
    if (!gauss_filter(w, h, params->gauss_filter_mask_size, ref, fref.data()) ||
        !gauss_filter(w, h, params->gauss_filter_mask_size, def, fdef.data()))
      return DICEGPU_ERR_ARG;
    ref = fref.data();
    def = fdef.data();
  }
  Ctx C;
  C.P = *params;
  std::vector<float> rgx((long)w * h), rgy((long)w * h), dgx, dgy;
  compute_gradients(w, h, ref, params->gradient_method, rgx.data(), rgy.data());
  C.ref.w = w; C.ref.h = h; C.ref.I = ref; C.ref.gx = rgx.data(); C.ref.gy = rgy.data();
  C.ref.has_gradients = true;
  C.def.w = w; C.def.h = h; C.def.I = def;
  if (params->use_def_gradients) {
    dgx.resize((long)w * h); dgy.resize((long)w * h);
    compute_gradients(w, h, def, params->gradient_method, dgx.data(), dgy.data());
    C.def.gx = dgx.data(); C.def.gy = dgy.data(); C.def.has_gradients = true;
  }
  Subset s;
  for (int i = 0; i < n; ++i) {
    const double* f = fields + (long)i * DICEGPU_FIELD_STRIDE;
    s.init_square((int)f[DICEGPU_F_COORD_X], (int)f[DICEGPU_F_COORD_Y], params->subset_size);
    s.init_ref(C.ref);
    ShapeFn sf;
    sf.init(C.P);
    sf.from_fields(f);
    gamma_out[i] = objective_gamma(C, s, sf, nullptr);
  }
  return 0;
}
