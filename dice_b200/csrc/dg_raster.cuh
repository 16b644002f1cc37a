// dg_raster.cuh -- conformal subset pixel lists built on the device.
//
// Each subset owns a set of shapes: boundary shapes (role 0), whose union
// makes the subset, and excluded shapes (role 1), whose pixels are removed.
// The pixel test of each shape is the reference's get_owned_pixels
// (DICe_Shape.cpp:136-219 circle, 259-279 rectangle, 322-420 polygon) with
// its float arithmetic kept: the circle compares float squares against
// radius^2, the polygon sums float atan2 angle differences wrapped against
// double pi (atan2 correctly rounded to float).  Pixels are emitted in (y, x) order over the union's bounding box,
// the order Subset(cx, cy, Conformal_Area_Def) builds (DICe_Subset.cpp:115-142).
//
// One warp per subset: the warp walks the bounding box a row at a time in
// 32-column steps, each lane tests one pixel, and a ballot gives every owned
// pixel its position.  A count pass sizes the lists, a fill pass writes them.
#pragma once
#include <cstdint>

#include "dicegpu.h"

struct RasterArgs {
  const dicegpu_shape* shapes;   // grouped by subset
  const int32_t* shape_off;      // [n + 1] into shapes
  const int32_t* vx;
  const int32_t* vy;
  int n;
  int32_t* counts;               // count pass: pixels per subset
  const int32_t* offsets;        // fill pass: [n + 1]
  int32_t* px;
  int32_t* py;
};

// angle_2d (DICe_Shape.cpp:87-102) in the reference's precision, with the
// float atan2 correctly rounded (the double atan2 rounded to float) so that
// pixels lying exactly on a polygon edge, whose edge term is +-pi, are
// decided the same way as on the host.
__device__ __forceinline__ float raster_angle(float x1, float y1, float x2, float y2) {
  const float t1 = (float)atan2((double)y1, (double)x1), t2 = (float)atan2((double)y2, (double)x2);
  float d = __fsub_rn(t2, t1);
  for (int k = 0; k < 4 && (double)d > 3.14159265358979323846; ++k) d = (float)((double)d - 6.28318530717958647692);
  for (int k = 0; k < 4 && (double)d < -3.14159265358979323846; ++k) d = (float)((double)d + 6.28318530717958647692);
  return d;
}

__device__ __forceinline__ bool raster_has(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, int x,
                                           int y) {
  if (s.kind == DICEGPU_SHAPE_CIRCLE) {
    // pixels more than radius + 1 away on an axis are outside; the early
    // exit keeps the integer squares below 2^31 for far excluded circles
    const int lim = (int)s.radius + 1;
    if (abs(x - s.cx) > lim || abs(y - s.cy) > lim) return false;
    const float r2 = __fmul_rn(s.radius, s.radius);
    const float dx = (float)((x - s.cx) * (x - s.cx)), dy = (float)((y - s.cy) * (y - s.cy));
    return __fadd_rn(dx, dy) <= r2;
  }
  if (s.kind == DICEGPU_SHAPE_RECTANGLE) {
    const int ox = s.cx - s.width / 2, oy = s.cy - s.height / 2;
    return x >= ox && x < ox + s.width && y >= oy && y < oy + s.height;
  }
  const int32_t* ax = vx + s.vertex_offset;
  const int32_t* ay = vy + s.vertex_offset;
  float angle = 0.0f;
  for (int i = 0; i < s.vertex_count; ++i) {
    const int j = (i + 1 == s.vertex_count) ? 0 : i + 1;
    angle = __fadd_rn(angle, raster_angle((float)(ax[i] - x), (float)(ay[i] - y), (float)(ax[j] - x),
                                          (float)(ay[j] - y)));
  }
  return (double)fabsf(angle) >= 3.14159265358979323846;
}

__device__ __forceinline__ void raster_box(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, int& x0,
                                           int& x1, int& y0, int& y1) {
  if (s.kind == DICEGPU_SHAPE_CIRCLE) {
    x0 = (int)__fsub_rn(__fsub_rn((float)s.cx, s.radius), 1.0f);
    x1 = (int)__fadd_rn(__fadd_rn((float)s.cx, s.radius), 1.0f);
    y0 = (int)__fsub_rn(__fsub_rn((float)s.cy, s.radius), 1.0f);
    y1 = (int)__fadd_rn(__fadd_rn((float)s.cy, s.radius), 1.0f);
  } else if (s.kind == DICEGPU_SHAPE_RECTANGLE) {
    x0 = s.cx - s.width / 2; x1 = x0 + s.width - 1;
    y0 = s.cy - s.height / 2; y1 = y0 + s.height - 1;
  } else {
    x0 = x1 = vx[s.vertex_offset];
    y0 = y1 = vy[s.vertex_offset];
    for (int i = 1; i < s.vertex_count; ++i) {
      x0 = min(x0, vx[s.vertex_offset + i]); x1 = max(x1, vx[s.vertex_offset + i]);
      y0 = min(y0, vy[s.vertex_offset + i]); y1 = max(y1, vy[s.vertex_offset + i]);
    }
  }
}

template <bool FILL>
__global__ void __launch_bounds__(256) raster_kernel(RasterArgs a) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < a.n; i += warps) {
    const int s0 = a.shape_off[i], s1 = a.shape_off[i + 1];
    int x0 = 0, x1 = -1, y0 = 0, y1 = -1;
    bool any = false;
    for (int k = s0; k < s1; ++k) {
      if (a.shapes[k].role != 0) continue;
      int bx0, bx1, by0, by1;
      raster_box(a.shapes[k], a.vx, a.vy, bx0, bx1, by0, by1);
      if (!any) { x0 = bx0; x1 = bx1; y0 = by0; y1 = by1; any = true; }
      else { x0 = min(x0, bx0); x1 = max(x1, bx1); y0 = min(y0, by0); y1 = max(y1, by1); }
    }
    int cnt = 0;
    const int base = FILL ? a.offsets[i] : 0;
    for (int y = y0; any && y <= y1; ++y)
      for (int xs = x0; xs <= x1; xs += 32) {
        const int x = xs + lane;
        bool own = false;
        if (x <= x1) {
          bool in = false, out = false;
          for (int k = s0; k < s1; ++k) {
            const dicegpu_shape& s = a.shapes[k];
            if (s.role == 0 ? in : out) continue;
            const bool h = raster_has(s, a.vx, a.vy, x, y);
            if (s.role == 0) in = h; else out = h;
          }
          own = in && !out;
        }
        const unsigned m = __ballot_sync(0xffffffffu, own);
        if (FILL && own) {
          const int pos = base + cnt + __popc(m & ((1u << lane) - 1u));
          a.px[pos] = x < 0 ? 0 : x;
          a.py[pos] = y < 0 ? 0 : y;
        }
        cnt += __popc(m);
      }
    if (!FILL && lane == 0) a.counts[i] = cnt;
  }
}
