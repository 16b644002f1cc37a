// dg_pass.cuh -- CTA-wide passes over the pixels of one subset, in the
// reference's floating-point arithmetic.
//
// One CTA of W warps (T = 32 W threads) owns one subset at a time; thread t
// takes subset pixels t, t + T, t + 2T, ...  A pass is Subset::initialize on
// the deformed image (DICe_Subset.cpp:390-426): map, round, border and mask
// tests, interpolation of the deformed image (and its gradients).  It keeps
// every pixel's values in shared memory (reference intensity F, deformed
// intensity G, gradients, stretched offsets, liveness), because the reference
// then forms sums that depend on each other in order:
//   * Subset::mean / gamma / contrast and Objective::sigma sum in float, one
//     pixel after the other (DICe_Subset.cpp:285-340, 597-620,
//     DICe_Objective.cpp:150-184): here one thread sums the stored values in
//     pixel order (chain_sum), the only way to get the same float;
//   * Objective_ZNSSD::computeUpdateFast (DICe_Objective.cpp:523-546) adds the
//     float products r_i r_j and GmF r_i, each rounded to float, into double
//     sums.  H = sum fl(r_i r_j) is formed as the exact products, summed by the
//     FP64 tensor core (mma.sync m8n8k4), minus the sum of the products'
//     rounding errors fma(r_i, r_j, -fl(r_i r_j)) (exact floats, summed per
//     thread in float and across threads in double), in a sweep over the
//     stored pixels (h_sweep) that runs while one thread sums the deformed
//     mean; q needs that mean, so a last sweep (q_sweep) adds fl(GmF r_i) in
//     double.
// Double sums are taken in another order than the reference's sequential one;
// that changes them in the last bits of a double (~1e-16 relative), far below
// the float rounding of the parameter update they feed.
#pragma once

#include <type_traits>

#include "dg_device.cuh"


namespace dg {

// Section timers of a profiling build (-DDG_PROFILE): cycles per section
// summed over all CTAs (thread 0's clock).  Compiled out otherwise.
#ifdef DG_PROFILE
static __device__ unsigned long long g_prof[16];   // per translation unit
#define DG_PT(var) const long long var = clock64()
#define DG_PACC_T(i, t0, thr)                                                               \
  do {                                                                                      \
    if (threadIdx.x == (thr)) atomicAdd(&g_prof[i], (unsigned long long)(clock64() - (t0))); \
  } while (0)
#define DG_PACC(i, t0) DG_PACC_T(i, t0, 0)
#else
#define DG_PT(var)
#define DG_PACC_T(i, t0, thr)
#define DG_PACC(i, t0)
#endif

template <int SHAPE>
struct Layout {
  static constexpr int NS = SHAPE == DICEGPU_QUADRATIC_SF ? 12 : 6;   // parameter slots
  static constexpr int VW = SHAPE == DICEGPU_QUADRATIC_SF ? 16 : 8;   // mma vector width (padded)
  static constexpr int VS = SHAPE == DICEGPU_QUADRATIC_SF ? 24 : 8;   // staging row stride (floats)
  static constexpr int NP = NS * (NS + 1) / 2;                        // products r_i r_j, i <= j
  static constexpr int NMAX = NS;
};

// index of the pair (i, j), i <= j, of the upper triangle in row order
__host__ __device__ constexpr int pair_index(int i, int j, int ns) { return i * ns - i * (i - 1) / 2 + (j - i); }

// ---------------------------------------------------------------------------
// Shared memory of a frame CTA
// ---------------------------------------------------------------------------
// Broadcast values and the Gauss-Newton solve's workspace (one per CTA).
struct __align__(16) Ctl {
  int work;                      // subset of this round
  int n, minx, maxx, miny, maxy; // live pixels and their box, last pass
  int status, conv, info;        // solve outcome
  int pad0;
  float fres[4];                 // chain results
  float slots[12];               // parameters after a solve step
  float upd_old[12];             // momentum: the previous update (compact order)
  float cond;
  float pad1[3];
  double red[8];                 // cta_sum's per-warp partial sums
  double q[12];
  int piv[12];
  // the Hessian (compact order, row major, then its LU factors) in the first
  // NS * NS entries, its inverse (column k written by lane k) in the next
  // NS * NS; the CTA's shared memory holds only the shape function's share
  double H[2 * 144];
};
// the inverse's place in Ctl::H
template <int SHAPE>
__device__ __forceinline__ double* ctl_inv(Ctl& c) {
  return c.H + Layout<SHAPE>::NS * Layout<SHAPE>::NS;
}

// Per-warp partial results of a pass.
template <int SHAPE>
struct __align__(16) WarpOut {
  double M[Layout<SHAPE>::VW * Layout<SHAPE>::VW];   // exact product sums
  double E[Layout<SHAPE>::NP];                       // rounding errors of the float products
  double q[Layout<SHAPE>::NS];                       // right-hand side (slot order)
  int n, minx, maxx, miny, maxy, pad[3];
};

// The Nelder-Mead state of Simplex::minimize (DICe_Simplex.cpp:60-277), one
// copy per warp: every warp runs the same bookkeeping on its own copy (lane 0
// writes, the warp reads after __syncwarp), so all warps take the same
// branches and evaluate the same points together.
struct __align__(16) SimplexState {
  float pts[13][12];
  float gv[13];
  float psum[12];
  float ptry[12];
  float init[12];
  float base[12];
};

__host__ __device__ inline size_t a16(size_t x) { return (x + 15) & ~(size_t)15; }
// per-pixel array capacity: a multiple of 32 pixels
__host__ __device__ inline int pix_cap(int npix_max) { return (npix_max + 31) & ~31; }
// distance between the per-pixel float arrays: cap + 4 floats, so that the
// same pixel's entries of the rows fall in distinct banks (and every row
// starts on a 16-byte boundary)
__host__ __device__ inline int pix_stride(int cap) { return cap + 4; }
// stored per-pixel rows besides F and G: the affine residual vector r_0..r_5,
// or the quadratic subset's gradients (its residuals are products of them)
// Stored rows of an affine subset (DG_AFF_ROWS): 6, its residual vector;
// 4, the gradients and the stretched offsets Dx, Dy; 2, the gradients only
// (the sweeps form the residuals from them).
#ifndef DG_AFF_ROWS
#define DG_AFF_ROWS 6
#endif
template <int SHAPE>
struct PixRows {
  static constexpr int NR = SHAPE == DICEGPU_QUADRATIC_SF ? 2 : DG_AFF_ROWS;
  // the sweeps read the residual vector straight from the rows
  static constexpr bool RESID = SHAPE != DICEGPU_QUADRATIC_SF && DG_AFF_ROWS == 6;
};
template <int SHAPE>
struct SmemPlan {
  // Ctl up to the shape function's share of H (Hessian and inverse)
  static __host__ __device__ size_t wout(int) {
    return a16(offsetof(Ctl, H) + 2 * sizeof(double) * Layout<SHAPE>::NS * Layout<SHAPE>::NS);
  }
  static __host__ __device__ size_t simplex(int W) { return wout(W) + a16((size_t)W * sizeof(WarpOut<SHAPE>)); }
  static __host__ __device__ size_t vbuf(int W) { return simplex(W) + a16((size_t)W * sizeof(SimplexState)); }
  // the sweeps' staging rows: only when the residual vectors are not stored
  static __host__ __device__ size_t pix(int W) {
    return vbuf(W) + (PixRows<SHAPE>::RESID ? 0 : a16((size_t)W * 32 * Layout<SHAPE>::VS * sizeof(float)));
  }
  // F, G and the stored rows (floats, pix_stride apart), then one byte per pixel
  static __host__ __device__ size_t pix_bytes(int cap) {
    return a16((size_t)(2 + PixRows<SHAPE>::NR) * pix_stride(cap) * 4 + (size_t)cap);
  }
  static __host__ __device__ size_t total(int W, int cap) { return pix(W) + pix_bytes(cap); }
};

extern __shared__ __align__(16) unsigned char dg_smem[];

__device__ __forceinline__ Ctl& ctl() { return *reinterpret_cast<Ctl*>(dg_smem); }
template <int SHAPE>
__device__ __forceinline__ WarpOut<SHAPE>* wouts() {
  return reinterpret_cast<WarpOut<SHAPE>*>(dg_smem + SmemPlan<SHAPE>::wout(blockDim.x >> 5));
}
template <int SHAPE>
__device__ __forceinline__ SimplexState& sx_state() {
  return reinterpret_cast<SimplexState*>(dg_smem + SmemPlan<SHAPE>::simplex(blockDim.x >> 5))[threadIdx.x >> 5];
}
template <int SHAPE>
__device__ __forceinline__ float* warp_vbuf() {
  return reinterpret_cast<float*>(dg_smem + SmemPlan<SHAPE>::vbuf(blockDim.x >> 5)) +
         (threadIdx.x >> 5) * 32 * Layout<SHAPE>::VS;
}

// The per-pixel arrays: F (reference intensity), G (deformed intensity, 0 at
// pixels that are not live), the rows R(i) (affine: the residual vector of
// the last Gauss-Newton pass, 0 at pixels that are not live; quadratic: the
// gradients; after a PK_STATE pass rows 0 and 1 hold the gradients), L (bit 0
// live: active and not deactivated this step; bit 1 active).  The arrays
// beyond the subset's pixels up to a multiple of 32 hold zeros after a pass.
struct PixArrays {
  float* F;
  float* G;
  float* R0;
  int S;        // float distance between rows
  uint8_t* L;
  __device__ __forceinline__ float* R(int i) const { return R0 + (size_t)i * S; }
};
// Where a CTA's pixel arrays live: its shared memory, or for subsets too
// large for it, this CTA's slice of a global scratch buffer (`stride` bytes
// per CTA).
template <int SHAPE>
__device__ __forceinline__ float* pix_base(unsigned char* scratch, size_t stride) {
  return scratch ? reinterpret_cast<float*>(scratch + (size_t)blockIdx.x * stride)
                 : reinterpret_cast<float*>(dg_smem + SmemPlan<SHAPE>::pix(blockDim.x >> 5));
}
template <int SHAPE>
__device__ __forceinline__ PixArrays pix_arrays_at(float* b, int cap) {
  PixArrays a;
  const int S = pix_stride(cap);
  a.S = S;
  a.F = b;
  a.G = b + S;
  a.R0 = b + 2 * (size_t)S;
  a.L = reinterpret_cast<uint8_t*>(b + (size_t)(2 + PixRows<SHAPE>::NR) * S);
  return a;
}

// ---------------------------------------------------------------------------
// CTA reductions and sequential float sums (fixed order: deterministic)
// ---------------------------------------------------------------------------
// CTA-wide double sum of one value per thread, the same in every thread.
// Uses Ctl's red[] as scratch; starts and ends with a barrier.
__device__ __forceinline__ double cta_sum(double v) {
  Ctl& c = ctl();
  v = warp_sum(v);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) c.red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  const int W = blockDim.x >> 5;
  for (int w = 0; w < W; ++w) s += c.red[w];
  __syncthreads();
  return s;
}
__device__ __forceinline__ int cta_sum_i(int v) {
  return (int)cta_sum((double)v);
}

// Sequential float sum a[0] + a[1] + ... + a[n-1] starting from 0.0f, each
// addition rounded: the reference's `sum += x` loop.  a is 16-byte aligned.
// Zeros stand for skipped pixels: adding +0.0f leaves every running sum
// unchanged (the sum, starting at +0.0f, is never -0.0f).  The next 16
// values are loaded while the current 16 are added, so the chain runs at the
// addition's latency rather than the shared-memory load's.
#define DG_ADD4(s, v)        \
  s = __fadd_rn(s, (v).x); \
  s = __fadd_rn(s, (v).y); \
  s = __fadd_rn(s, (v).z); \
  s = __fadd_rn(s, (v).w)
static __device__ __noinline__ float chain_sum(const float* a, int n, float s = 0.0f) {
  const float4* a4 = reinterpret_cast<const float4*>(a);
  const int nq = n >> 2;
  int q = 0;
  if (nq >= 4) {
    float4 v0 = a4[0], v1 = a4[1], v2 = a4[2], v3 = a4[3];
    for (q = 4; q + 4 <= nq; q += 4) {
      const float4 w0 = a4[q], w1 = a4[q + 1], w2 = a4[q + 2], w3 = a4[q + 3];
      DG_ADD4(s, v0); DG_ADD4(s, v1); DG_ADD4(s, v2); DG_ADD4(s, v3);
      v0 = w0; v1 = w1; v2 = w2; v3 = w3;
    }
    DG_ADD4(s, v0); DG_ADD4(s, v1); DG_ADD4(s, v2); DG_ADD4(s, v3);
  }
  for (; q < nq; ++q) {
    const float4 v = a4[q];
    DG_ADD4(s, v);
  }
  for (int i = nq << 2; i < n; ++i) s = __fadd_rn(s, a[i]);
  return s;
}

// The same over the pixels whose liveness byte has `bit` set (the others
// count as +0.0f); a and m are 16- and 4-byte aligned.
__device__ __forceinline__ float4 masked4(float4 v, uchar4 b, unsigned bit) {
  return make_float4((b.x & bit) ? v.x : 0.0f, (b.y & bit) ? v.y : 0.0f, (b.z & bit) ? v.z : 0.0f,
                     (b.w & bit) ? v.w : 0.0f);
}
static __device__ __noinline__ float chain_sum_masked(const float* a, const uint8_t* m, unsigned bit, int n) {
  float s = 0.0f;
  const float4* a4 = reinterpret_cast<const float4*>(a);
  const uchar4* m4 = reinterpret_cast<const uchar4*>(m);
  const int nq = n >> 2;
  int q = 0;
  if (nq >= 4) {
    float4 v0 = masked4(a4[0], m4[0], bit), v1 = masked4(a4[1], m4[1], bit);
    float4 v2 = masked4(a4[2], m4[2], bit), v3 = masked4(a4[3], m4[3], bit);
    for (q = 4; q + 4 <= nq; q += 4) {
      const float4 w0 = masked4(a4[q], m4[q], bit), w1 = masked4(a4[q + 1], m4[q + 1], bit);
      const float4 w2 = masked4(a4[q + 2], m4[q + 2], bit), w3 = masked4(a4[q + 3], m4[q + 3], bit);
      DG_ADD4(s, v0); DG_ADD4(s, v1); DG_ADD4(s, v2); DG_ADD4(s, v3);
      v0 = w0; v1 = w1; v2 = w2; v3 = w3;
    }
    DG_ADD4(s, v0); DG_ADD4(s, v1); DG_ADD4(s, v2); DG_ADD4(s, v3);
  }
  for (; q < nq; ++q) {
    const float4 v = masked4(a4[q], m4[q], bit);
    DG_ADD4(s, v);
  }
  for (int i = nq << 2; i < n; ++i) s = __fadd_rn(s, (m[i] & bit) ? a[i] : 0.0f);
  return s;
}
#undef DG_ADD4

// Up to four chains at once (lanes 0..k-1 of warp 0, in lockstep), chain i
// over the pixels whose liveness byte in m has a bit of byte i of `bits` set
// (all pixels when m is null); results in every thread.  Barriers before
// (the arrays are complete) and after.
__device__ __forceinline__ void chains(int k, const float* a0, const float* a1, const float* a2, const float* a3,
                                       const uint8_t* m, unsigned bits, int n, float* out) {
  Ctl& c = ctl();
  __syncthreads();
  if (threadIdx.x < k) {
    const float* a = threadIdx.x == 0 ? a0 : threadIdx.x == 1 ? a1 : threadIdx.x == 2 ? a2 : a3;
    const unsigned bit = (bits >> (8 * threadIdx.x)) & 0xffu;
    c.fres[threadIdx.x] = m ? chain_sum_masked(a, m, bit, n) : chain_sum(a, n);
  }
  __syncthreads();
  for (int i = 0; i < k; ++i) out[i] = c.fres[i];
  __syncthreads();
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

// ---------------------------------------------------------------------------
// Pass inputs
// ---------------------------------------------------------------------------
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
  int cap;         // per-pixel array capacity
  float* pix;      // the CTA's per-pixel arrays (pix_base)
};

// What a MASKED pass reads besides: this subset's mask descriptor
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

// Pixel coordinates of pixel p of a subset (clamped at 0 as the Subset
// constructors do, DICe_Subset.cpp:66-68, :100-101).
struct PixelWalk {
  int side, x0, y0, row, col, drow, dcol;
  bool square;
  __device__ __forceinline__ PixelWalk(const PassIn& in, int first, int step) {
    square = in.off < 0;
    side = 2 * in.half + 1;
    x0 = in.cx - in.half;
    y0 = in.cy - in.half;
    row = col = drow = dcol = 0;
    if (square) {
      row = first / side; col = first - row * side;
      drow = step / side; dcol = step - drow * side;
    }
  }
  __device__ __forceinline__ void xy(const PassIn& in, int p, int& x, int& y) const {
    if (square) {
      x = max(x0 + col, 0);
      y = max(y0 + row, 0);
    } else {
      x = max(__ldg(in.px + in.off + p), 0);
      y = max(__ldg(in.py + in.off + p), 0);
    }
  }
  __device__ __forceinline__ void advance() {
    if (square) {
      col += dcol; row += drow;
      if (col >= side) { col -= side; ++row; }
    }
  }
};

// Kinds of pass:
//   PK_GN    : the Gauss-Newton iteration's initialisation: gradients, every
//              per-pixel array (the sums follow in h_sweep and q_sweep)
//   PK_STATE : deformed-state initialisation with gradients (sigma's state)
//   PK_GAMMA : intensities only (gamma, simplex evaluations)
enum { PK_GN = 0, PK_STATE = 1, PK_GAMMA = 2 };

// One pass (Subset::initialize on the deformed image).  Ends with the live
// count and box in Ctl (all threads may read them after the final barrier).
template <int SHAPE, int INTERP, bool DEFGRAD, int KIND, bool MASKED>
__device__ __forceinline__ void cta_pass(const PassInT<MASKED> in, const MapConst k) {
  using L = Layout<SHAPE>;
  constexpr bool GRADS = KIND != PK_GAMMA;
  constexpr bool AFF = SHAPE != DICEGPU_QUADRATIC_SF;
  const int tid = threadIdx.x, T = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const bool use_ref_grads = !DEFGRAD;
  const float fcx = (float)in.cx, fcy = (float)in.cy;
  const int W = in.def.w, H = in.def.h;
  const PixArrays A = pix_arrays_at<SHAPE>(in.pix, in.cap);
  int n = 0;
  int minx = in.cx, maxx = in.cx, miny = in.cy, maxy = in.cy;
  MaskView mv;
  if constexpr (MASKED) mv = MaskView(in.mdesc, in.mbits, in.bpoly, in.bvx, in.bvy);
  PixelWalk pw(in, tid, T);
  const int npad = (in.npix + 31) & ~31;
  for (int p = tid; p < npad; p += T) {
    if (p >= in.npix) {
      // the padding up to a multiple of 32 pixels: zeros for the sweeps
      A.G[p] = 0.0f;
      A.L[p] = 0;
      if (KIND == PK_GN) {
#pragma unroll
        for (int i = 0; i < PixRows<SHAPE>::NR; ++i) A.R(i)[p] = 0.0f;
      }
      continue;
    }
    int x, y;
    pw.xy(in, p, x, y);
    pw.advance();
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
    float mx, my, Dx, Dy;
    const float dxf = __fsub_rn((float)x, fcx), dyf = __fsub_rn((float)y, fcy);
    map_offset<SHAPE>(k, dxf, dyf, fcx, fcy, mx, my, Dx, Dy);
    const int px = round_pixel(mx), py = round_pixel(my);
    // 4-pixel border deactivation (DICe_Subset.cpp:408)
    bool live = active && !(px < 4 || px >= W - 4 || py < 4 || py >= H - 4);
    if (MASKED && live) live = !mv.hides(px, py);
    float G = 0.0f, gx = 0.0f, gy = 0.0f;
    if (live) {
      if (GRADS && DEFGRAD) interp_ref<INTERP, true>(in.def, mx, my, G, gx, gy);
      else interp_ref<INTERP, false>(in.def, mx, my, G, gx, gy);
      if (GRADS && !DEFGRAD) {
        gx = rin ? __ldg(in.refgx + ri) : 0.0f;
        gy = rin ? __ldg(in.refgy + ri) : 0.0f;
      }
      ++n;
      minx = min(minx, x); maxx = max(maxx, x);
      miny = min(miny, y); maxy = max(maxy, y);
    }
    A.F[p] = F;
    A.G[p] = live ? G : 0.0f;
    A.L[p] = (uint8_t)((live ? 1 : 0) | (active ? 2 : 0));
    if (KIND == PK_GN && PixRows<SHAPE>::RESID) {
      // the residual vector of Objective_ZNSSD::computeUpdateFast (:538)
      float r[L::VW];
#pragma unroll
      for (int i = 0; i < L::VW; ++i) r[i] = 0.0f;
      if (live) residuals_D<SHAPE>(k, dxf, dyf, Dx, Dy, gx, gy, use_ref_grads, r);
#pragma unroll
      for (int i = 0; i < PixRows<SHAPE>::NR; ++i) A.R(i)[p] = r[i];
    } else if (GRADS) {
      A.R(0)[p] = gx;
      A.R(1)[p] = gy;
      if (KIND == PK_GN && AFF && PixRows<SHAPE>::NR == 4) {
        A.R(2)[p] = Dx;
        A.R(3)[p] = Dy;
      }
    }
  }
  // per-warp results
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
    int nn = 0, a0 = in.cx, a1 = in.cx, b0 = in.cy, b1 = in.cy;
    const int NW = T >> 5;
    for (int w = 0; w < NW; ++w) {
      nn += all[w].n;
      a0 = min(a0, all[w].minx); a1 = max(a1, all[w].maxx);
      b0 = min(b0, all[w].miny); b1 = max(b1, all[w].maxy);
    }
    cl.n = nn; cl.minx = a0; cl.maxx = a1; cl.miny = b0; cl.maxy = b1;
  }
  __syncthreads();
}

// The residual vector of a stored pixel formed from its stored gradients
// (Quadratic_Shape_Function::residuals, :580-614; the affine one, :350-396,
// with the stretched offsets stored or formed again as the pass formed them).
template <int SHAPE>
__device__ __forceinline__ void stored_residuals(const PassIn& in, const PixArrays& A, const MapConst& k, int p, int x,
                                                 int y, bool use_ref_grads, float* r) {
  const float dxf = __fsub_rn((float)x, (float)in.cx), dyf = __fsub_rn((float)y, (float)in.cy);
  if (SHAPE == DICEGPU_QUADRATIC_SF) {
    residuals_D<SHAPE>(k, dxf, dyf, dxf, dyf, A.R(0)[p], A.R(1)[p], use_ref_grads, r);
  } else {
    float Dx, Dy;
    if (PixRows<SHAPE>::NR >= 4) {
      Dx = A.R(2)[p];
      Dy = A.R(3)[p];
    } else {
      affine_D(k, dxf, dyf, Dx, Dy);
    }
    residuals_D<SHAPE>(k, dxf, dyf, Dx, Dy, A.R(0)[p], A.R(1)[p], use_ref_grads, r);
  }
}

// The Hessian sweep over the stored pixels, run by warps w0 .. w0 + nw - 1
// (full warps, 32 pixels a step): the exact products r_i r_j summed by the
// FP64 mma (WarpOut.M) and the float products' rounding errors
// fma(r_i, r_j, -fl(r_i r_j)) (WarpOut.E), whose difference is the
// reference's sum of float products.  The affine residual rows are read
// straight from the stored arrays (rows pix_stride apart: conflict-free
// fragments); quadratic residuals are formed from the stored gradients and
// staged.  Warps outside the range return at once.  No barrier.
template <int SHAPE, bool DEFGRAD>
__device__ __forceinline__ void h_sweep(const PassIn in, const MapConst k, int w0, int nw) {
  using L = Layout<SHAPE>;
  constexpr bool AFF = SHAPE != DICEGPU_QUADRATIC_SF;
  constexpr bool ROWS = PixRows<SHAPE>::RESID;   // residual vectors stored per pixel
  constexpr int NSET = 2;   // independent mma accumulator sets
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (warp < w0 || warp >= w0 + nw) return;
  const bool use_ref_grads = !DEFGRAD;
  const PixArrays A = pix_arrays_at<SHAPE>(in.pix, in.cap);
  double c[NSET][3][2];
#pragma unroll
  for (int s2 = 0; s2 < NSET; ++s2)
#pragma unroll
    for (int b = 0; b < 3; ++b) { c[s2][b][0] = 0.0; c[s2][b][1] = 0.0; }
  float e[L::NP];
#pragma unroll
  for (int i = 0; i < L::NP; ++i) e[i] = 0.0f;
  const int nblk = (in.npix + 31) >> 5;
  const int kk = lane & 3, ii = lane >> 2;
  // stored residual rows: the mma fragment's row (residual index ii, zero
  // beyond the six)
  const float* frag = A.R(ROWS && ii < PixRows<SHAPE>::NR ? ii : 0) + kk;
  const unsigned vbase = (unsigned)__cvta_generic_to_shared(warp_vbuf<SHAPE>());
  PixelWalk pw(in, (warp - w0) * 32 + lane, 32 * nw);
  for (int blk = warp - w0; blk < nblk; blk += nw) {
    const int p = blk * 32 + lane;
    float v[L::VW];
#pragma unroll
    for (int i = 0; i < L::VW; ++i) v[i] = 0.0f;
    if (A.L[p] & 1) {
      if (ROWS) {
#pragma unroll
        for (int i = 0; i < L::NS; ++i) v[i] = A.R(i)[p];
      } else {
        int x, y;
        pw.xy(in, p, x, y);
        stored_residuals<SHAPE>(in, A, k, p, x, y, use_ref_grads, v);
      }
      int idx = 0;
#pragma unroll
      for (int i = 0; i < L::NS; ++i)
#pragma unroll
        for (int j = i; j < L::NS; ++j, ++idx) {
          const float pr = __fmul_rn(v[i], v[j]);
          e[idx] = __fadd_rn(e[idx], fmaf(v[i], v[j], -pr));
        }
    }
    if (!ROWS) {
      pw.advance();
      // stage the warp's 32 pixel vectors
      const unsigned vrow = vbase + (unsigned)(lane * L::VS) * 4u;
#pragma unroll
      for (int i = 0; i < L::VW; i += 4) sts_v4(vrow + 4u * i, v[i], v[i + 1], v[i + 2], v[i + 3]);
      __syncwarp();
    }
    // groups of 4 pixels through the FP64 mma
#pragma unroll
    for (int g = 0; g < 8; ++g) {
      double(&cs)[3][2] = c[g % NSET];
      if (ROWS) {
        const double a0 = ii < PixRows<SHAPE>::NR ? (double)frag[blk * 32 + 4 * g] : 0.0;
        dmma_8x8x4(cs[0][0], cs[0][1], a0, a0);
      } else {
        const unsigned src = vbase + (unsigned)((4 * g + kk) * L::VS + ii) * 4u;
        const double a0 = (double)lds_f(src);
        dmma_8x8x4(cs[0][0], cs[0][1], a0, a0);
        if (!AFF) {
          const double a1 = (double)lds_f(src + 32u);
          dmma_8x8x4(cs[1][0], cs[1][1], a0, a1);
          dmma_8x8x4(cs[2][0], cs[2][1], a1, a1);
        }
      }
    }
    if (!ROWS) __syncwarp();
  }
#pragma unroll
  for (int s2 = 1; s2 < NSET; ++s2)
#pragma unroll
    for (int b = 0; b < 3; ++b) {
      c[0][b][0] += c[s2][b][0];
      c[0][b][1] += c[s2][b][1];
    }
  // the accumulator fragments into the warp's dense symmetric matrix
  WarpOut<SHAPE>& wo = wouts<SHAPE>()[warp];
  const int r = lane >> 2, cc = 2 * (lane & 3);
  constexpr int VW = L::VW;
  double* C = wo.M;
  const double(&cf)[3][2] = c[0];
  if (!AFF) {
    C[r * VW + cc] = cf[0][0];           C[r * VW + cc + 1] = cf[0][1];
    C[r * VW + 8 + cc] = cf[1][0];       C[r * VW + 8 + cc + 1] = cf[1][1];
    C[(8 + cc) * VW + r] = cf[1][0];     C[(8 + cc + 1) * VW + r] = cf[1][1];
    C[(8 + r) * VW + 8 + cc] = cf[2][0]; C[(8 + r) * VW + 8 + cc + 1] = cf[2][1];
  } else {
    C[r * VW + cc] = cf[0][0];
    C[r * VW + cc + 1] = cf[0][1];
  }
#pragma unroll
  for (int i = 0; i < L::NP; ++i) {
    const double sm = warp_sum((double)e[i]);
    if (lane == 0) wo.E[i] = sm;
  }
}

// The right-hand side sweep: q_i = sum over live pixels of fl(GmF * r_i) in
// double, GmF = (G - meanG) - (F - meanF) in float (DICe_Objective.cpp:
// 528-537), by nt threads of whole warps, this one the vt-th.  Per-warp sums
// go to WarpOut.q.  No barrier.
template <int SHAPE, bool DEFGRAD>
__device__ __forceinline__ void q_sweep(const PassIn in, const MapConst k, float meanG, float meanF, int vt, int nt) {
  using L = Layout<SHAPE>;
  constexpr bool ROWS = PixRows<SHAPE>::RESID;
  const int lane = threadIdx.x & 31;
  const bool use_ref_grads = !DEFGRAD;
  const PixArrays A = pix_arrays_at<SHAPE>(in.pix, in.cap);
  double q[L::NS];
#pragma unroll
  for (int i = 0; i < L::NS; ++i) q[i] = 0.0;
  PixelWalk pw(in, vt, nt);
  for (int p = vt; p < in.npix; p += nt) {
    if (A.L[p] & 1) {
      const float GmF = __fsub_rn(__fsub_rn(A.G[p], meanG), __fsub_rn(A.F[p], meanF));
      float r[L::VW];
      if (ROWS) {
#pragma unroll
        for (int i = 0; i < L::NS; ++i) r[i] = A.R(i)[p];
      } else {
        int x, y;
        pw.xy(in, p, x, y);
        stored_residuals<SHAPE>(in, A, k, p, x, y, use_ref_grads, r);
      }
#pragma unroll
      for (int i = 0; i < L::NS; ++i) q[i] = __dadd_rn(q[i], (double)__fmul_rn(GmF, r[i]));
    }
    if (!ROWS) pw.advance();
  }
  WarpOut<SHAPE>& wo = wouts<SHAPE>()[threadIdx.x >> 5];
#pragma unroll
  for (int i = 0; i < L::NS; ++i) {
    const double sm = warp_sum(q[i]);
    if (lane == 0) wo.q[i] = sm;
  }
}

}  // namespace dg
