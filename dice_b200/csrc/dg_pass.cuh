// dg_pass.cuh -- one warp-wide pass over the pixels of a subset.
//
// The hot loop of the path: Subset::initialize on the deformed image
// (DICe_Subset.cpp:390-426) fused with the Gauss-Newton accumulation of
// Objective_ZNSSD::computeUpdateFast (DICe_Objective.cpp:523-546) or with the
// intensity moments of Subset::gamma (DICe_Subset.cpp:323-340).  It is a
// separate non-inlined function taking everything it reads by value, so its
// register allocation does not compete with the per-subset control code.
#pragma once

#include <type_traits>

#include "dg_device.cuh"

namespace dg {

// Section timers of a profiling build (-DDG_PROFILE): warp cycles per section
// summed over all warps.  Compiled out otherwise.
#ifdef DG_PROFILE
static __device__ unsigned long long g_prof[8];   // per translation unit
#define DG_PT(var) const long long var = clock64()
#define DG_PACC(i, t0)                                                                    \
  do {                                                                                    \
    if ((threadIdx.x & 31) == 0) atomicAdd(&g_prof[i], (unsigned long long)(clock64() - (t0))); \
  } while (0)
#else
#define DG_PT(var)
#define DG_PACC(i, t0)
#endif

template <int SHAPE>
struct Layout {
  static constexpr int NS = SHAPE == DICEGPU_QUADRATIC_SF ? 12 : 6;   // parameter slots
  static constexpr int VW = SHAPE == DICEGPU_QUADRATIC_SF ? 16 : 8;   // [r, d, 1] padded
  static constexpr int VS = SHAPE == DICEGPU_QUADRATIC_SF ? 24 : 8;   // smem row stride (conflict-free)
  static constexpr int ID = NS;        // column of d = G - F
  static constexpr int IONE = NS + 1;  // column of 1
  static constexpr int NMAX = NS;
};

// Pixels per lane per step of a pass: each step maps, interpolates and
// stages 32 * DG_PPL pixels before the mma accumulation, so that the tap
// loads of DG_PPL independent pixels are in flight together.
#ifndef DG_PPL
#define DG_PPL 1
#endif
constexpr int PPL = DG_PPL;
// independent FP64 mma accumulator sets of the affine pass
#ifndef DG_NSET_AFFINE
#define DG_NSET_AFFINE 2
#endif

template <int SHAPE>
struct __align__(16) WarpSmem {
  float vbuf[32 * PPL * Layout<SHAPE>::VS];
  double M[Layout<SHAPE>::VW * Layout<SHAPE>::VW];
};

// Dynamic shared memory of the frame kernel: one WarpSmem per warp.  Taken
// from the extern array in every user so the compiler keeps shared-space
// (not generic) addressing.
extern __shared__ __align__(16) unsigned char dg_smem[];

template <int SHAPE>
__device__ __forceinline__ WarpSmem<SHAPE>* warp_smem() {
  return reinterpret_cast<WarpSmem<SHAPE>*>(dg_smem) + (threadIdx.x >> 5);
}

__device__ __forceinline__ void sts_v4(unsigned addr, float a, float b, float c, float d) {
  asm volatile("st.shared.v4.f32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "f"(a), "f"(b), "f"(c), "f"(d)
               : "memory");
}
__device__ __forceinline__ float lds_f(unsigned addr) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(v) : "r"(addr) : "memory");
  return v;
}

// Result of one pass over the subset pixels.
struct PassOut {
  int n;                    // active pixels
  double sumF;              // sum of F over active pixels (shifted by K)
  double sumFall;           // sum of F over all subset pixels (shifted; Gauss-Newton passes)
  double sG, sG2, sF2, sGF; // shifted moments (gamma passes)
  double sgx2, sgy2;        // sum of unrotated gradient^2 (sigma)
  int minx, maxx, miny, maxy;
};

// Everything a pass reads, passed by value.
struct PassIn {
  DevImage def;
  const float* __restrict__ refI;
  const float* __restrict__ refgx;
  const float* __restrict__ refgy;
  int refw;
  long reflim;
  const int32_t* __restrict__ px;
  const int32_t* __restrict__ py;
  int half;        // square half-width (lists: unused)
  int cx, cy, npix, off;
  float K;         // intensity shift for the moment sums
};

// What a MASKED pass reads besides (the unmasked passes get the plain
// PassIn, which the call passes by value): this subset's mask descriptor
// (obstruction box x0, y0, w, h, word offset; blocked polygon count and
// table offset), the obstruction words, the blocked-polygon table (vertex
// offset, count, box x0, x1, y0, y1 per polygon), the polygons' vertices,
// and for evolving subsets the list pixels' evolution state (0 inactive, 1
// active, 2 active with the reference intensity in pfv; nullptr otherwise).
struct PassInMasked : PassIn {
  const int32_t* __restrict__ mdesc;
  const uint32_t* __restrict__ mbits;
  const int32_t* __restrict__ bpoly;
  const int32_t* __restrict__ bvx;
  const int32_t* __restrict__ bvy;
  const uint8_t* pflag;
  const float* pfv;
};
template <bool MASKED>
using PassInT = typename std::conditional<MASKED, PassInMasked, PassIn>::type;

// Whether pixel (px, py) is set in the mask box (x0, y0, w, h) at words.
__device__ __forceinline__ bool mask_bit(const uint32_t* __restrict__ words, int x0, int y0, int w, int h,
                                         int px, int py) {
  const unsigned dx = (unsigned)(px - x0), dy = (unsigned)(py - y0);
  if (dx >= (unsigned)w || dy >= (unsigned)h) return false;
  const unsigned long bit = (unsigned long)dy * (unsigned)w + dx;
  return (__ldg(words + (bit >> 5)) >> (bit & 31)) & 1u;
}

// One subset's masks, unpacked from its descriptor.
struct MaskView {
  int ox, oy, ow, oh;                 // obstruction box
  const uint32_t* __restrict__ bits;  // its words
  int np;                             // blocked polygons
  const int32_t* __restrict__ poly;   // their table rows
  const int32_t* __restrict__ bvx;
  const int32_t* __restrict__ bvy;

  __device__ __forceinline__ MaskView()
      : ox(0), oy(0), ow(0), oh(0), bits(nullptr), np(0), poly(nullptr), bvx(nullptr), bvy(nullptr) {}
  __device__ __forceinline__ MaskView(const int32_t* md, const uint32_t* mbits, const int32_t* bpoly,
                                      const int32_t* vx, const int32_t* vy)
      : ox(md[0]), oy(md[1]), ow(md[2]), oh(md[3]), bits(mbits + md[4]), np(md[5]), poly(bpoly + 6 * md[6]),
        bvx(vx), bvy(vy) {}

  // is_obstructed_pixel, then the blocked-pixel test, at the rounded mapped
  // pixel (Subset::initialize, DICe_Subset.cpp:412-422): an obstruction bit,
  // or inside a blocker's deformed boundary (box first)
  __device__ __forceinline__ bool hides(int px, int py) const {
    if (mask_bit(bits, ox, oy, ow, oh, px, py)) return true;
    for (int q = 0; q < np; ++q) {
      const int32_t* pd = poly + 6 * q;
      if (px < __ldg(pd + 2) || px > __ldg(pd + 3) || py < __ldg(pd + 4) || py > __ldg(pd + 5)) continue;
      const int vo = __ldg(pd);
      if (polygon_has(bvx + vo, bvy + vo, __ldg(pd + 1), px, py)) return true;
    }
    return false;
  }
};

//   ACC_H   : accumulate sum v v^T into the warp's smem matrix (Gauss-Newton)
//   GRADS   : interpolate the deformed gradients (DEFGRAD) / read reference ones
//   MOMENTS : FP64 intensity moments for gamma
//   MASKED  : also deactivate pixels whose position rounds into the
//             subset's obstruction bitmap or a blocked polygon (Subset::initialize,
//             DICe_Subset.cpp:412-422); for positive coordinates, which the
//             border test leaves, is_obstructed_pixel's rounding is the
//             border test's
template <int SHAPE, int INTERP, bool DEFGRAD, bool ACC_H, bool GRADS, bool MOMENTS, bool MASKED>
__device__ __noinline__ PassOut subset_pass(const PassInT<MASKED> in, const MapConst k) {
  using L = Layout<SHAPE>;
  const int lane = threadIdx.x & 31;
  const bool use_ref_grads = !DEFGRAD;
  const float fcx = (float)in.cx, fcy = (float)in.cy;
  const int W = in.def.w, H = in.def.h;
  PassOut o;
  int n = 0;
  // per-lane partial sums: FP32 over this lane's pixels (the reference sums
  // these in FP32 over the whole subset), FP64 across the warp; the gamma
  // moments are FP64 throughout
  float sumF = 0.0f, sgx2 = 0.0f, sgy2 = 0.0f, sumFall = 0.0f;
  double sG = 0.0, sG2 = 0.0, sF2 = 0.0, sGF = 0.0, sFd = 0.0;
  int minx = in.cx, maxx = in.cx, miny = in.cy, maxy = in.cy;
  // independent accumulator sets (pixel group g goes to set g % NSET) so that
  // consecutive mma instructions do not wait on each other
  constexpr int NSET = SHAPE == DICEGPU_QUADRATIC_SF ? 2 : DG_NSET_AFFINE;
  double c[NSET][3][2];
#pragma unroll
  for (int s2 = 0; s2 < NSET; ++s2)
#pragma unroll
    for (int b = 0; b < 3; ++b) { c[s2][b][0] = 0.0; c[s2][b][1] = 0.0; }
  // square subsets: (row, col) of this lane's pixel advanced by 32 per step
  const int side = 2 * in.half + 1;
  int row = 0, col = 0, drow = 0, dcol = 0;
  if (in.off < 0) {
    row = lane / side; col = lane - row * side;
    drow = 32 / side; dcol = 32 - drow * side;
  }
  const int x0 = in.cx - in.half, y0 = in.cy - in.half;
  MaskView mv;
  if constexpr (MASKED) mv = MaskView(in.mdesc, in.mbits, in.bpoly, in.bvx, in.bvy);
  const unsigned vbase = (unsigned)__cvta_generic_to_shared(warp_smem<SHAPE>()->vbuf);
  for (int base = 0; base < in.npix; base += 32 * PPL) {
    float vv[PPL][L::VW];
#pragma unroll
    for (int u = 0; u < PPL; ++u) {
    float* v = vv[u];
    const int p = base + 32 * u + lane;
#pragma unroll
    for (int i = 0; i < L::VW; ++i) v[i] = 0.0f;
    int x = 0, y = 0;
    if (in.off < 0) {
      x = max(x0 + col, 0);   // Subset ctors clamp negative coordinates (DICe_Subset.cpp:66-68, :100-101)
      y = max(y0 + row, 0);
      col += dcol; row += drow;
      if (col >= side) { col -= side; ++row; }
    } else if (p < in.npix) {
      x = max(__ldg(in.px + in.off + p), 0);
      y = max(__ldg(in.py + in.off + p), 0);
    }
    if (p < in.npix) {
      float mx, my, Dx, Dy;
      const float dxf = __fsub_rn((float)x, fcx), dyf = __fsub_rn((float)y, fcy);
      map_offset<SHAPE>(k, dxf, dyf, fcx, fcy, mx, my, Dx, Dy);
      const int px = round_pixel(mx), py = round_pixel(my);
      // the reference reads intensities_[y*w+x] unchecked (row-major wrap);
      // same element inside the array, 0 outside it
      const long ri = (long)y * in.refw + x;
      const bool rin = ri < in.reflim;
      float F = rin ? __ldg(in.refI + ri) : 0.0f;
      // subset evolution: an inactive pixel takes no part; a turned-on one
      // has its stored reference intensity
      bool active = true;
      if constexpr (MASKED) {
        if (in.pflag) {
          const int st = in.pflag[in.off + p];
          active = st != 0;
          if (st == 2) F = in.pfv[in.off + p];
        }
      }
      if (ACC_H && active) sumFall += F - in.K;
      // 4-pixel border deactivation (DICe_Subset.cpp:408)
      bool live = active && !(px < 4 || px >= W - 4 || py < 4 || py >= H - 4);
      if (MASKED && live) live = !mv.hides(px, py);
      if (live) {
        float G, gx = 0.0f, gy = 0.0f;
        if (GRADS && DEFGRAD) interp_interior<INTERP, true>(in.def, mx, my, G, gx, gy);
        else interp_interior<INTERP, false>(in.def, mx, my, G, gx, gy);
        if (GRADS && !DEFGRAD) {
          gx = rin ? __ldg(in.refgx + ri) : 0.0f;
          gy = rin ? __ldg(in.refgy + ri) : 0.0f;
        }
        ++n;
        const float Fs = F - in.K, Gs = G - in.K;
        if (MOMENTS) {
          sFd += (double)Fs;
          sG += (double)Gs;
          sG2 = fma((double)Gs, (double)Gs, sG2);
          sF2 = fma((double)Fs, (double)Fs, sF2);
          sGF = fma((double)Gs, (double)Fs, sGF);
        } else {
          sumF += Fs;
        }
        if (GRADS) {
          sgx2 = fmaf(gx, gx, sgx2);
          sgy2 = fmaf(gy, gy, sgy2);
          minx = min(minx, x); maxx = max(maxx, x);
          miny = min(miny, y); maxy = max(maxy, y);
        }
        if (ACC_H) {
          residuals_D<SHAPE>(k, dxf, dyf, Dx, Dy, gx, gy, use_ref_grads, v);
          v[L::ID] = G - F;
          v[L::IONE] = 1.0f;
        }
      }
    }
    }
    if (ACC_H) {
      // stage the 32 * PPL pixel vectors, then groups of 4 pixels through the FP64 mma
#pragma unroll
      for (int u = 0; u < PPL; ++u) {
        const unsigned vrow = vbase + (unsigned)((32 * u + lane) * L::VS) * 4u;
#pragma unroll
        for (int i = 0; i < L::VW; i += 4)
          sts_v4(vrow + 4u * i, vv[u][i], vv[u][i + 1], vv[u][i + 2], vv[u][i + 3]);
      }
      __syncwarp();
      const int kk = lane & 3, ii = lane >> 2;
#pragma unroll
      for (int g = 0; g < 8 * PPL; ++g) {
        const unsigned src = vbase + (unsigned)((4 * g + kk) * L::VS + ii) * 4u;
        double(&cs)[3][2] = c[g % NSET];
        if (SHAPE == DICEGPU_QUADRATIC_SF) {
          const double a0 = (double)lds_f(src), a1 = (double)lds_f(src + 32u);
          dmma_8x8x4(cs[0][0], cs[0][1], a0, a0);
          dmma_8x8x4(cs[1][0], cs[1][1], a0, a1);
          dmma_8x8x4(cs[2][0], cs[2][1], a1, a1);
        } else {
          const double a0 = (double)lds_f(src);
          dmma_8x8x4(cs[0][0], cs[0][1], a0, a0);
        }
      }
      __syncwarp();
    }
  }
#pragma unroll
  for (int s2 = 1; s2 < NSET; ++s2)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      c[0][b][0] += c[s2][b][0];
      c[0][b][1] += c[s2][b][1];
    }
  o.n = warp_sum_i(n);
  o.sumF = MOMENTS ? warp_sum(sFd) : warp_sum((double)sumF);
  o.sumFall = ACC_H ? warp_sum((double)sumFall) : 0.0;
  if (MOMENTS) {
    o.sG = warp_sum(sG); o.sG2 = warp_sum(sG2); o.sF2 = warp_sum(sF2); o.sGF = warp_sum(sGF);
  } else {
    o.sG = o.sG2 = o.sF2 = o.sGF = 0.0;
  }
  if (GRADS) {
    o.sgx2 = warp_sum((double)sgx2); o.sgy2 = warp_sum((double)sgy2);
    o.minx = warp_min_i(minx); o.maxx = warp_max_i(maxx);
    o.miny = warp_min_i(miny); o.maxy = warp_max_i(maxy);
  } else {
    o.sgx2 = o.sgy2 = 0.0;
    o.minx = o.maxx = in.cx; o.miny = o.maxy = in.cy;
  }
  if (ACC_H) {
    // scatter the accumulator fragments into the warp's dense symmetric matrix
    double* C = warp_smem<SHAPE>()->M;
    __syncwarp();
    const int r = lane >> 2, cc = 2 * (lane & 3);
    constexpr int VW = L::VW;
    const double(&cf)[3][2] = c[0];
    if (SHAPE == DICEGPU_QUADRATIC_SF) {
      C[r * VW + cc] = cf[0][0];           C[r * VW + cc + 1] = cf[0][1];
      C[r * VW + 8 + cc] = cf[1][0];       C[r * VW + 8 + cc + 1] = cf[1][1];
      C[(8 + cc) * VW + r] = cf[1][0];     C[(8 + cc + 1) * VW + r] = cf[1][1];
      C[(8 + r) * VW + 8 + cc] = cf[2][0]; C[(8 + r) * VW + 8 + cc + 1] = cf[2][1];
    } else {
      C[r * VW + cc] = cf[0][0];
      C[r * VW + cc + 1] = cf[0][1];
    }
    __syncwarp();
  }
  return o;
}

}  // namespace dg
