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
//
// Masks: a subset pixel is deactivated when its deformed position rounds
// into the subset's obstruction bitmap (static, from its obstructed shapes)
// or into one of its blocked polygons (rebuilt before each tracking wave
// from the deformed boundaries of its blocking subsets).  Each subset has a
// descriptor of DG_MASK_DESC ints: the obstruction box (x0, y0, w, h, word
// offset; a box of width 0 is no mask; bit (y - y0) * w + (x - x0) of the
// words from the offset is pixel (x, y)) and the blocked polygons (count,
// offset in the polygon table).
//
// Subset evolution (Subset::turn_on_previously_obstructed_pixels): the
// excluded pixels then stay in the lists, inactive, as the reference's
// conformal Subset keeps them with is_active false (DICe_Subset.cpp:155-160).
#pragma once
#include <climits>
#include <cstdint>

#include "dg_device.cuh"
#include "dicegpu.h"

// polygons of the blocking subsets of one blocked subset (shared memory)
#define DG_MAX_BLOCK_POLYS 64

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
  const double* fields;          // subset centroids (squares)
  int square_half;               // half side of the square of a subset without boundary, -1: empty
  // subset evolution: excluded pixels stay in the lists with state 0 (the
  // others 1); the count pass also counts the active pixels
  int keep_excluded;
  uint8_t* flags;                // fill pass
  int32_t* active;               // count pass
};

// the winding test of a closed vertex loop (dg::polygon_has, dg_device.cuh)
__device__ __forceinline__ bool raster_polygon_has(const int32_t* ax, const int32_t* ay, int nv, int x, int y) {
  return dg::polygon_has(ax, ay, nv, x, y);
}

// get_owned_pixels' test, or deactivate_pixels' (excluded: the circle adds
// its integer squares before converting them)
__device__ __forceinline__ bool raster_has(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, int x,
                                           int y, bool excluded = false) {
  if (s.kind == DICEGPU_SHAPE_CIRCLE) {
    // pixels more than radius + 1 away on an axis are outside; the early
    // exit keeps the integer squares below 2^31 for far excluded circles
    const int lim = (int)s.radius + 1;
    if (abs(x - s.cx) > lim || abs(y - s.cy) > lim) return false;
    const float r2 = __fmul_rn(s.radius, s.radius);
    const int ix = (x - s.cx) * (x - s.cx), iy = (y - s.cy) * (y - s.cy);
    if (excluded) return (float)(ix + iy) <= r2;
    return __fadd_rn((float)ix, (float)iy) <= r2;
  }
  if (s.kind == DICEGPU_SHAPE_RECTANGLE) {
    const int ox = s.cx - s.width / 2, oy = s.cy - s.height / 2;
    return x >= ox && x < ox + s.width && y >= oy && y < oy + s.height;
  }
  return raster_polygon_has(vx + s.vertex_offset, vy + s.vertex_offset, s.vertex_count, x, y);
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
      if (a.shapes[k].role != DICEGPU_ROLE_BOUNDARY) continue;
      int bx0, bx1, by0, by1;
      raster_box(a.shapes[k], a.vx, a.vy, bx0, bx1, by0, by1);
      if (!any) { x0 = bx0; x1 = bx1; y0 = by0; y1 = by1; any = true; }
      else { x0 = min(x0, bx0); x1 = max(x1, bx1); y0 = min(y0, by0); y1 = max(y1, by1); }
    }
    // a subset without boundary shapes: the square Subset(cx, cy, w, h)
    // (DICe_Subset.cpp:78-101), every pixel owned
    const bool square = !any && a.square_half >= 0;
    if (square) {
      const double* f = a.fields + (size_t)i * DICEGPU_FIELD_STRIDE;
      const int cx = (int)f[DICEGPU_F_COORD_X], cy = (int)f[DICEGPU_F_COORD_Y];
      x0 = cx - a.square_half; x1 = cx + a.square_half;
      y0 = cy - a.square_half; y1 = cy + a.square_half;
    }
    int cnt = 0, nact = 0;
    const int base = FILL ? a.offsets[i] : 0;
    for (int y = y0; (any || square) && y <= y1; ++y)
      for (int xs = x0; xs <= x1; xs += 32) {
        const int x = xs + lane;
        bool own = false, act = false;
        if (x <= x1) {
          if (square) {
            own = act = true;
          } else {
            // excluded shapes test the clamped coordinates, as
            // deactivate_pixels sees the constructed (clamped) pixel list
            const int ex = x < 0 ? 0 : x, ey = y < 0 ? 0 : y;
            bool in = false, out = false;
            for (int k = s0; k < s1; ++k) {
              const dicegpu_shape& s = a.shapes[k];
              if (s.role == DICEGPU_ROLE_BOUNDARY) {
                if (!in) in = raster_has(s, a.vx, a.vy, x, y);
              } else if (s.role == DICEGPU_ROLE_EXCLUDED) {
                if (!out) out = raster_has(s, a.vx, a.vy, ex, ey, true);
              }
            }
            own = in && (!out || a.keep_excluded);
            act = in && !out;
          }
        }
        const unsigned m = __ballot_sync(0xffffffffu, own);
        if (FILL && own) {
          const int pos = base + cnt + __popc(m & ((1u << lane) - 1u));
          a.px[pos] = x < 0 ? 0 : x;
          a.py[pos] = y < 0 ? 0 : y;
          if (a.flags) a.flags[pos] = act ? 1 : 0;
        }
        cnt += __popc(m);
        nact += __popc(__ballot_sync(0xffffffffu, act));
      }
    if (!FILL && lane == 0) {
      a.counts[i] = cnt;
      if (a.active) a.active[i] = nact;
    }
  }
}

// Obstruction bitmaps: the owned pixels of each listed subset's obstructed
// shapes (Subset ctor, DICe_Subset.cpp:162-167), over the box of its
// descriptor.  The words are zero on entry.  One warp per subset.
struct ObstArgs {
  const dicegpu_shape* shapes;
  const int32_t* shape_off;
  const int32_t* vx;
  const int32_t* vy;
  const int32_t* list;   // subsets with obstructed shapes
  int nlist;
  const int32_t* desc;
  uint32_t* bits;
};

__global__ void __launch_bounds__(256) obstruction_kernel(ObstArgs a) {
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < a.nlist; t += warps) {
    const int i = a.list[t];
    const int32_t* d = a.desc + (size_t)i * DG_MASK_DESC;
    const int bx = d[0], by = d[1], bw = d[2], bh = d[3];
    uint32_t* words = a.bits + d[4];
    const int s0 = a.shape_off[i], s1 = a.shape_off[i + 1];
    for (int y = by; y < by + bh; ++y)
      for (int x = bx + lane; x < bx + bw; x += 32) {
        bool on = false;
        for (int k = s0; k < s1 && !on; ++k)
          if (a.shapes[k].role == DICEGPU_ROLE_OBSTRUCTED) on = raster_has(a.shapes[k], a.vx, a.vy, x, y);
        if (on) {
          const long bit = (long)(y - by) * bw + (x - bx);
          atomicOr(words + (bit >> 5), 1u << (bit & 31));
        }
      }
  }
}

// Blocked polygons of the blocked subsets of one tracking wave
// (Schema::check_for_blocking_subsets, DICe_Schema.cpp:4529-4557): for every
// conformal blocker j, each boundary polygon or rectangle mapped by j's
// parameters about j's centroid, rounded, and stretched by the skin factor
// about its integer vertex centroid (get_owned_pixels with a shape function,
// DICe_Shape.cpp:136-219, 322-396), stored with its vertex box in the
// subset's slots of the polygon table; the masked pass tests pixels against
// them.  Blocker j's parameters come from the live fields when j precedes
// the blocked subset in index order (it has run in an earlier wave), from
// the frame-start snapshot otherwise.  One warp per blocked subset.
struct BlockArgs {
  dg::DevParams P;
  const dicegpu_shape* shapes;
  const int32_t* shape_off;
  const int32_t* vx;
  const int32_t* vy;
  const double* fields;     // live
  const double* snapshot;   // at frame start
  const int32_t* blk_off;   // blockers of subset i: blk_ids[blk_off[i] .. blk_off[i+1])
  const int32_t* blk_ids;
  const uint8_t* conformal; // subset has boundary shapes
  const int32_t* list;      // blocked subsets of this wave
  int nlist;
  const int32_t* dv_off;    // per subset: offset of its deformed vertices
  const int32_t* dp_off;    // per subset: offset of its polygons in the table
  int32_t* dvx;
  int32_t* dvy;
  int32_t* polys;           // 6 ints per polygon: vertex offset, count, x0, x1, y0, y1
  int32_t* desc;
  float skin;
};

template <int SHAPE>
__global__ void __launch_bounds__(256) blocked_kernel(BlockArgs a) {
  using namespace dg;
  const int lane = threadIdx.x & 31;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; t < a.nlist; t += warps) {
    const int i = a.list[t];
    int npoly = 0, wpos = a.dv_off[i];
    const int pbase = a.dp_off[i];
    for (int b = a.blk_off[i]; b < a.blk_off[i + 1]; ++b) {
      const int j = a.blk_ids[b];
      if (!a.conformal[j]) continue;   // a square blocker covers nothing
      const double* f = (j < i ? a.fields : a.snapshot) + (size_t)j * DICEGPU_FIELD_STRIDE;
      float slots[12];
      if (SHAPE == DICEGPU_QUADRATIC_SF) {
        for (int q = 0; q < 12; ++q) slots[q] = (float)f[DICEGPU_F_QUAD_A + q];
      } else {
        for (int q = 0; q < 12; ++q) slots[q] = 0.0f;
        for (int q = 0; q < a.P.N; ++q) slots[a.P.slot[q]] = (float)f[DICEGPU_F_DISP_X + a.P.slot[q]];
      }
      const float fcx = (float)(int)f[DICEGPU_F_COORD_X], fcy = (float)(int)f[DICEGPU_F_COORD_Y];
      MapConst k;
      make_mapconst<SHAPE>(slots, false, fcx, fcy, k);
      for (int m = a.shape_off[j]; m < a.shape_off[j + 1]; ++m) {
        const dicegpu_shape& s = a.shapes[m];
        if (s.role != DICEGPU_ROLE_BOUNDARY || npoly >= DG_MAX_BLOCK_POLYS) continue;
        const int nv = s.kind == DICEGPU_SHAPE_RECTANGLE ? 4 : s.vertex_count;
        const int ox = s.cx - s.width / 2, oy = s.cy - s.height / 2;
        long long sx = 0, sy = 0;
        for (int v = lane; v < nv; v += 32) {
          int x, y;
          if (s.kind == DICEGPU_SHAPE_RECTANGLE) {
            x = (v == 1 || v == 2) ? ox + s.width : ox;
            y = (v >= 2) ? oy + s.height : oy;
          } else {
            x = a.vx[s.vertex_offset + v];
            y = a.vy[s.vertex_offset + v];
          }
          float mx, my, Dx, Dy;
          map_offset<SHAPE>(k, __fsub_rn((float)x, fcx), __fsub_rn((float)y, fcy), fcx, fcy, mx, my, Dx, Dy);
          int nx = (int)mx, ny = (int)my;
          if (__fsub_rn(mx, (float)nx) >= 0.5f) ++nx;
          if (__fsub_rn(my, (float)ny) >= 0.5f) ++ny;
          a.dvx[wpos + v] = nx;
          a.dvy[wpos + v] = ny;
          sx += nx;
          sy += ny;
        }
        for (int o = 16; o > 0; o >>= 1) {
          sx += __shfl_xor_sync(0xffffffffu, sx, o);
          sy += __shfl_xor_sync(0xffffffffu, sy, o);
        }
        const int ccx = (int)((double)sx / (double)nv), ccy = (int)((double)sy / (double)nv);
        int x0 = INT_MAX, x1 = INT_MIN, y0 = INT_MAX, y1 = INT_MIN;
        for (int v = lane; v < nv; v += 32) {
          const int nx = (int)__fadd_rn(__fmul_rn(a.skin, (float)(a.dvx[wpos + v] - ccx)), (float)ccx);
          const int ny = (int)__fadd_rn(__fmul_rn(a.skin, (float)(a.dvy[wpos + v] - ccy)), (float)ccy);
          a.dvx[wpos + v] = nx;
          a.dvy[wpos + v] = ny;
          x0 = min(x0, nx); x1 = max(x1, nx); y0 = min(y0, ny); y1 = max(y1, ny);
        }
        for (int o = 16; o > 0; o >>= 1) {
          x0 = min(x0, __shfl_xor_sync(0xffffffffu, x0, o));
          x1 = max(x1, __shfl_xor_sync(0xffffffffu, x1, o));
          y0 = min(y0, __shfl_xor_sync(0xffffffffu, y0, o));
          y1 = max(y1, __shfl_xor_sync(0xffffffffu, y1, o));
        }
        if (lane == 0) {
          int32_t* pd = a.polys + 6 * (size_t)(pbase + npoly);
          pd[0] = wpos; pd[1] = nv; pd[2] = x0; pd[3] = x1; pd[4] = y0; pd[5] = y1;
        }
        ++npoly;
        wpos += nv;
      }
    }
    if (lane == 0) {
      int32_t* d = a.desc + (size_t)i * DG_MASK_DESC;
      d[5] = npoly;
      d[6] = pbase;
    }
  }
}
