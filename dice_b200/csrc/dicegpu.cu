// dicegpu.cu -- kernels and C ABI of libdicegpu.so (sm_100a).
//
// Kernels
//   gradient_kernel   Image_::compute_gradients (finite difference, optional
//                     5x5 smoothing), DICe_Image.cpp:1015-1093
//   frame_kernel      persistent work-stealing correlation of every subset:
//                     one CTA per subset (dg_frame.cuh; instantiated in
//                     frame_inst.cu)
//   interp_kernel     Image_::interpolate_*_all at arbitrary points
// The C ABI (include/dicegpu.h) owns device memory and launches on the
// caller's stream; it never throws and never falls back to the CPU.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <map>
#include <mutex>
#include <vector>

#include "dg_frame.cuh"
#include "dg_adjoint.cuh"
#include "dg_raster.cuh"
#include "dg_vsg.cuh"
#include "dicegpu.h"

using namespace dg;

// consecutive subsets per work-queue chunk (0: two per warp of a CTA)
#ifndef DG_QUEUE_CHUNK
#define DG_QUEUE_CHUNK 0
#endif

// ---------------------------------------------------------------------------
// gradients
// ---------------------------------------------------------------------------
// Finite differences with c1 = 1/12, c2 = -8/12 stored as float
// (DICe_Image.cpp:214-215), one-sided within two pixels of the border.
// Separate rounded products and sums (no contraction) so that the result is
// bit-identical to the reference's expression order.
__global__ void gradient_fd_kernel(int w, int h, const float* __restrict__ I, float* __restrict__ gx,
                                   float* __restrict__ gy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w || y >= h) return;
  const float c1 = (float)(1.0 / 12.0), c2 = (float)(-8.0 / 12.0);
  const size_t i = (size_t)y * w + x;
  float a, b;
  if (x < 2) a = __fsub_rn(I[i + 1], I[i]);
  else if (x >= w - 2) a = __fsub_rn(I[i], I[i - 1]);
  else a = __fsub_rn(__fsub_rn(__fadd_rn(__fmul_rn(c1, I[i - 2]), __fmul_rn(c2, I[i - 1])),
                               __fmul_rn(c2, I[i + 1])),
                     __fmul_rn(c1, I[i + 2]));
  if (y < 2) b = __fsub_rn(I[i + w], I[i]);
  else if (y >= h - 2) b = __fsub_rn(I[i], I[i - w]);
  else b = __fsub_rn(__fsub_rn(__fadd_rn(__fmul_rn(c1, I[i - 2 * (size_t)w]), __fmul_rn(c2, I[i - w])),
                               __fmul_rn(c2, I[i + w])),
                     __fmul_rn(c1, I[i + 2 * (size_t)w]));
  gx[i] = a;
  gy[i] = b;
}

// smooth_gradients_convolution_5_point (DICe_Image.cpp:1034-1060): outer
// product of (1,4,6,4,1)/16 on the interior, borders copied.
__global__ void gradient_smooth_kernel(int w, int h, const float* __restrict__ tx,
                                       const float* __restrict__ ty, float* __restrict__ gx,
                                       float* __restrict__ gy) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= w || y >= h) return;
  const size_t i = (size_t)y * w + x;
  if (x < 2 || x >= w - 2 || y < 2 || y >= h - 2) {
    gx[i] = tx[i];
    gy[i] = ty[i];
    return;
  }
  const float k[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
  float vx = 0.0f, vy = 0.0f;
#pragma unroll
  for (int a = 0; a < 5; ++a)
#pragma unroll
    for (int b = 0; b < 5; ++b) {
      const float c = __fmul_rn(k[a], k[b]);
      const size_t j = (size_t)(y + a - 2) * w + x + b - 2;
      vx = __fadd_rn(vx, __fmul_rn(c, tx[j]));
      vy = __fadd_rn(vy, __fmul_rn(c, ty[j]));
    }
  gx[i] = vx;
  gy[i] = vy;
}

// Image_::gauss_filter (DICe_Image.cpp:1194-1230).  The M x M weights travel
// by value in the parameter bank (uniform reads); each CTA stages its
// (32 + M - 1) x (8 + M - 1) input tile in shared memory.  The sum runs x
// offset outer, y offset inner, with every float product and sum rounded
// separately, as the reference's loop does; pixels within M/2+1 of an edge
// keep their value.
struct GaussWeights {
  float c[13 * 13];
};

constexpr int kGaussBX = 32, kGaussBY = 8, kGaussMaxTile = (kGaussBX + 12) * (kGaussBY + 12);

__global__ void __launch_bounds__(kGaussBX * kGaussBY)
gauss_filter_kernel(int w, int h, int M, const GaussWeights wt, const float* __restrict__ in,
                    float* __restrict__ out) {
  __shared__ float tile[kGaussMaxTile];
  const int R = M / 2;                 // taps reach R pixels either side
  const int half = M / 2 + 1;          // the reference's interior test
  const int TW = kGaussBX + 2 * R, TH = kGaussBY + 2 * R;
  const int x0 = blockIdx.x * kGaussBX - R, y0 = blockIdx.y * kGaussBY - R;
  const int tid = threadIdx.y * kGaussBX + threadIdx.x;
  for (int k = tid; k < TW * TH; k += kGaussBX * kGaussBY) {
    const int ty = k / TW, tx = k - ty * TW;
    const int gx = x0 + tx, gy = y0 + ty;
    tile[k] = (gx >= 0 && gx < w && gy >= 0 && gy < h) ? in[(size_t)gy * w + gx] : 0.0f;
  }
  __syncthreads();
  const int x = blockIdx.x * kGaussBX + threadIdx.x;
  const int y = blockIdx.y * kGaussBY + threadIdx.y;
  if (x >= w || y >= h) return;
  const size_t o = (size_t)y * w + x;
  if (!(x >= half && x < w - half && y >= half && y < h - half)) {
    out[o] = in[o];
    return;
  }
  float v = 0.0f;
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < M; ++j)
      v = __fadd_rn(v, __fmul_rn(wt.c[i * M + j], tile[(threadIdx.y + j) * TW + threadIdx.x + i]));
  out[o] = v;
}

// Incremental formulation (DICe_Schema.cpp:1671-1675, 1775-1789): a frame
// after the first starts with DISPLACEMENT_X / _Y at 0 and ends with them
// set to the accumulated displacement.
__global__ void incr_begin_kernel(double* __restrict__ fields, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  fields[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_DISP_X] = 0.0;
  fields[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_DISP_Y] = 0.0;
}
__global__ void incr_end_kernel(double* __restrict__ fields, double* __restrict__ acc, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double* f = fields + (size_t)i * DICEGPU_FIELD_STRIDE;
  acc[2 * i] += f[DICEGPU_F_DISP_X];
  acc[2 * i + 1] += f[DICEGPU_F_DISP_Y];
  f[DICEGPU_F_DISP_X] = acc[2 * i];
  f[DICEGPU_F_DISP_Y] = acc[2 * i + 1];
}
// The tracking routine re-reads every reference intensity from the new
// reference each incremental frame (DICe_Schema.cpp:1757-1759): turned-on
// pixels keep is_active and lose their stored intensity.
__global__ void evo_rebase_kernel(uint8_t* __restrict__ state, size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && state[i] == 2) state[i] = 1;
}

// (I, Gx, Gy) -> interleaved float4 (the layout the frame kernel gathers from)
__global__ void pack_kernel(size_t n, const float* __restrict__ I, const float* __restrict__ gx,
                            const float* __restrict__ gy, float4* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = make_float4(I[i], gx[i], gy[i], 0.0f);
}

// ---------------------------------------------------------------------------
// interpolation at arbitrary points (the Image_ interface), in the
// reference's arithmetic and border semantics: bilinear outside its range is
// 0; Keys-4 and bicubic compute the bilinear value near the border and then
// overwrite it with the kernel sum (DICe_Image.cpp:851-857, :496-502), whose
// taps are read through the row-major linear index.  Where that index leaves
// the image the reference reads past its array; here such taps read 0.
// ---------------------------------------------------------------------------
__device__ float lin_at(const float* a, long idx, long lim) {
  return (idx >= 0 && idx < lim) ? a[idx] : 0.0f;
}

// Image_::interpolate_bilinear (DICe_Image.cpp:432-445) on one channel
__device__ float bilinear_pt(const float* a, int w, int h, float lx, float ly) {
  if (lx < 0.0f || (double)lx >= w - 1.5 || ly < 0.0f || (double)ly >= h - 1.5) return 0.0f;
  const int x1 = (int)lx, x2 = x1 + 1, y1 = (int)ly, y2 = y1 + 1;
  return a[y1 * w + x1] * (x2 - lx) * (y2 - ly) + a[y1 * w + x2] * (lx - x1) * (y2 - ly) +
         a[y2 * w + x2] * (lx - x1) * (ly - y1) + a[y2 * w + x1] * (x2 - lx) * (ly - y1);
}

// one channel of the Keys-4 sum (cc = wy * wx in float, m outer, n inner)
__device__ float keys_pt(const float* a, int w, long lim, int ix, int iy, const float wx[6], const float wy[6]) {
  float v = 0.0f;
  for (int m = 0; m < 6; ++m) {
    const long r0 = (long)(iy - 2 + m) * w + ix - 2;
    for (int k = 0; k < 6; ++k) v = v + (wy[m] * wx[k]) * lin_at(a, r0 + k, lim);
  }
  return v;
}

// one channel of the bicubic polynomial (the expanded order of dg::bicubic_eval)
__device__ float bicubic_pt(const float* a, int w, long lim, int x0, int y0, float x, float y) {
  float f[4][4];
  for (int n = 0; n < 4; ++n)
    for (int m = 0; m < 4; ++m) f[n][m] = lin_at(a, (long)(y0 - 1 + m) * w + x0 - 1 + n, lim);
  return bicubic_eval(f, x, y);
}

__global__ void interp_kernel(int method, int w, int h, const float* __restrict__ I,
                              const float* __restrict__ gxi, const float* __restrict__ gyi, int n,
                              const float* __restrict__ xy, float* __restrict__ oi,
                              float* __restrict__ ogx, float* __restrict__ ogy) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const float lx = xy[2 * t], ly = xy[2 * t + 1];
  const bool grad = gxi && gyi && ogx && ogy;
  const long lim = (long)w * h;
  float v = 0.0f, a = 0.0f, b = 0.0f;
  if (method == DICEGPU_BILINEAR) {
    v = bilinear_pt(I, w, h, lx, ly);
    if (grad) { a = bilinear_pt(gxi, w, h, lx, ly); b = bilinear_pt(gyi, w, h, lx, ly); }
  } else if (method == DICEGPU_KEYS_FOURTH) {
    const int ix = (int)lx, iy = (int)ly;
    float wx[6], wy[6];
    keys_weights_ref_general(lx - (float)ix, wx);
    keys_weights_ref_general(ly - (float)iy, wy);
    v = keys_pt(I, w, lim, ix, iy, wx, wy);
    if (grad) { a = keys_pt(gxi, w, lim, ix, iy, wx, wy); b = keys_pt(gyi, w, lim, ix, iy, wx, wy); }
  } else {
    const int x0 = (int)lx, y0 = (int)ly;
    const float x = lx - (float)x0, y = ly - (float)y0;
    v = bicubic_pt(I, w, lim, x0, y0, x, y);
    if (grad) { a = bicubic_pt(gxi, w, lim, x0, y0, x, y); b = bicubic_pt(gyi, w, lim, x0, y0, x, y); }
  }
  oi[t] = v;
  if (grad) { ogx[t] = a; ogy[t] = b; }
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------
// upper bound on the persistent grid (and on its per-CTA queue heads)
static const int kMaxQueues = 8192;

template <typename T>
static int grow(T** p, size_t* cap, size_t need);

// A device array that only grows (contents are not kept across growth).
template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  int ensure(size_t n) { return grow(&p, &cap, n); }
  void release() { cudaFree(p); p = nullptr; cap = 0; }
};

struct dicegpu_ctx {
  dicegpu_params params;
  DevParams dp;
  int device = 0;
  int num_sms = 0;
  int smem_optin = 0;   // largest dynamic shared memory a CTA may opt in to
  // per-pixel arrays of subsets too large for shared memory: one slice per CTA
  bool pix_in_global = false;
  size_t pix_stride = 0;
  DevBuf<unsigned char> d_pix_scratch;
  cudaStream_t stream = nullptr;
  int W = 0, H = 0;
  float* d_ref = nullptr;
  float* d_ref_gx = nullptr;
  float* d_ref_gy = nullptr;
  float* d_def = nullptr;
  float* d_def_gx = nullptr;
  float* d_def_gy = nullptr;
  float* d_tmp = nullptr;   // smoothing scratch (2 planes)
  float4* d_def4 = nullptr; // deformed (I, Gx, Gy, 0) interleaved
  size_t img_cap = 0;       // pixels allocated per plane
  bool has_ref = false, has_def = false;
  int n = 0;
  size_t fields_cap = 0;
  double* d_fields = nullptr;
  int32_t* d_offsets = nullptr;
  int32_t* d_px = nullptr;
  int32_t* d_py = nullptr;
  size_t list_cap = 0, offs_cap = 0;
  bool use_lists = false;
  int list_npix_max = 0;    // largest pixel list (use_lists)
  uint8_t* d_force = nullptr;
  size_t force_cap = 0;
  bool use_force = false;
  int* d_counter = nullptr;
  int* d_status = nullptr;
  int32_t* d_passes = nullptr;
  size_t passes_cap = 0;
  double* d_unc = nullptr;   // uncertainty fields (params.compute_uncertainty)
  size_t unc_cap = 0;
  int unc_n = 0;             // subset count the buffer was zeroed for (0: invalid)
  int frame_index = 0;
  int warps_per_cta = 4;   // warps of the CTA that solves one subset
  int ctas_per_sm = 0;   // 0: occupancy-derived
  bool shape_set = false;  // the caller (or the autotuner) chose the launch shape
  // occupancy of the eight-warp shape, for the last kernel and shared memory asked
  const void* wide_fn = nullptr;
  size_t wide_smem = 0;
  int wide_per_sm = 0;
  int queue_mode = 1;    // 1: per-CTA queues with stealing, 0: one global queue
  int carveout = -1;     // preferred shared-memory carveout (percent), -1: driver default
  int chunk = DG_QUEUE_CHUNK;   // queue chunk (consecutive subsets); 0: 2 per warp of a CTA
  long long launches = 0;
  // captured frame sequence
  cudaStream_t cap_stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  long long graph_launches = 0;   // kernels per replay
  // conformal shapes (dicegpu_set_subset_shapes), grouped by subset
  std::vector<dicegpu_shape> h_shapes;
  std::vector<int32_t> h_shape_off, h_svx, h_svy;
  std::vector<uint8_t> h_conformal;
  DevBuf<dicegpu_shape> d_shapes;
  DevBuf<int32_t> d_shape_off, d_svx, d_svy;
  DevBuf<uint8_t> d_conformal;
  // pixel masks: descriptors (host copy kept), obstruction words, blocked words
  std::vector<int32_t> h_mask_desc;
  DevBuf<int32_t> d_mask_desc;
  DevBuf<uint32_t> d_mask_bits;
  bool use_masks = false;
  // subset evolution (params.use_subset_evolution, tracking routine): the
  // list pixels' state and stored reference intensities, their initial
  // state (restored at the first frame of a sequence) and per-subset active
  // counts
  bool has_evo = false;
  bool evo_suspend = false;   // the autotuner's trial frames leave the state alone
  size_t evo_total = 0;       // list pixels (state entries)
  DevBuf<uint8_t> d_pix_flag, d_pix_flag0;
  DevBuf<float> d_pix_f;
  DevBuf<int32_t> d_evo_nact, d_evo_nact0;
  // incremental formulation: accumulated DISPLACEMENT_X / _Y per subset, and
  // the reference planes a captured sequence restarts from
  DevBuf<double> d_acc;
  DevBuf<float> d_ref_saved;
  bool blocking_desc_ready = false;   // descriptors on the device for the tracking waves
  // blocking subsets and the tracking waves
  bool has_blocking = false;
  std::vector<int32_t> h_blk_off, h_blk_ids;
  DevBuf<int32_t> d_blk_off, d_blk_ids;
  std::vector<uint8_t> h_has_polys;   // blocked subsets with conformal blockers
  DevBuf<int32_t> d_dv_off, d_dvx, d_dvy, d_dp_off, d_bpoly;
  // neighbour initialization: NEIGHBOR_ID per subset (empty: none)
  std::vector<int32_t> h_neigh;
  DevBuf<int32_t> d_neigh;
  // Dependency waves, one plan per kind (bit 0: blocking subsets of the
  // tracking routine, bit 1: neighbour initialization): wave L is
  // d_wave[wave_off[L] ..) in index order, its blocked subsets d_bwave[bwave_off[L] ..)
  struct Plan {
    bool valid = false;
    std::vector<int32_t> wave_off, bwave_off;
    DevBuf<int32_t> d_wave, d_bwave;
  } plans[4];
  DevBuf<double> d_snapshot;
  int n_blocked = 0;                   // subsets with a conformal blocker
  // forced simplex: the caller's flags and the blocking rule's
  std::vector<uint8_t> h_force_user, h_force_block;
  std::vector<uint8_t> h_skip_user;   // dicegpu_set_skip_solve
  // VSG strain: the neighbour grid of the subset centres (rebuilt when the
  // window or the coordinates change) and the results
  int vsg_window = 0;
  int vsg_ncx = 0, vsg_ncy = 0;
  float vsg_x0 = 0.0f, vsg_y0 = 0.0f, vsg_cell = 1.0f, vsg_r2 = 0.0f;
  DevBuf<int32_t> d_vsg_cell_off, d_vsg_cell_pts, d_vsg_pos;
  DevBuf<float4> d_vsg_packed;
  DevBuf<int32_t> d_vsg_nbr;   // k nearest neighbours per subset (negative windows)
  DevBuf<double> d_vsg;
  std::vector<double> h_vsg_coords;   // the coordinates the grid was built for
};

// A failed runtime call returns DICEGPU_ERR_CUDA and clears the runtime's
// pending (non-sticky) error, so that it is not reported by a later check.
#define CK(x)                                  \
  do {                                         \
    cudaError_t e_ = (x);                      \
    if (e_ != cudaSuccess) {                   \
      cudaGetLastError();                      \
      return DICEGPU_ERR_CUDA;                 \
    }                                          \
  } while (0)

static bool gauss_weights(int M, GaussWeights& g);

static int build_devparams(const dicegpu_params& p, DevParams& d) {
  if (!p.enable_translation) return DICEGPU_ERR_ARG;
  if (p.shape_function != DICEGPU_AFFINE_SF && p.shape_function != DICEGPU_QUADRATIC_SF)
    return DICEGPU_ERR_UNSUPPORTED;
  if (p.interpolation < DICEGPU_BILINEAR || p.interpolation > DICEGPU_KEYS_FOURTH) return DICEGPU_ERR_ARG;
  if (!(p.optimization == DICEGPU_SIMPLEX || p.optimization == DICEGPU_GRADIENT_BASED ||
        p.optimization == DICEGPU_SIMPLEX_THEN_GRADIENT_BASED ||
        p.optimization == DICEGPU_GRADIENT_BASED_THEN_SIMPLEX))
    return DICEGPU_ERR_UNSUPPORTED;
  if (p.max_solver_iterations_fast < 0 || p.max_solver_iterations_robust < 1) return DICEGPU_ERR_ARG;
  if (p.correlation_routine != DICEGPU_GENERIC_ROUTINE && p.correlation_routine != DICEGPU_TRACKING_ROUTINE)
    return DICEGPU_ERR_ARG;
  if (!(std::fabs(p.obstruction_skin_factor) < 1.0e6)) return DICEGPU_ERR_ARG;
  if (p.initialization_method != DICEGPU_USE_FIELD_VALUES && p.initialization_method != DICEGPU_USE_NEIGHBOR_VALUES &&
      p.initialization_method != DICEGPU_USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY)
    return DICEGPU_ERR_UNSUPPORTED;
  if (p.gauss_filter_images) {
    GaussWeights g;
    if (!gauss_weights(p.gauss_filter_mask_size, g)) return DICEGPU_ERR_ARG;
  }
  std::memset(&d, 0, sizeof(d));
  d.shape = p.shape_function;
  if (d.shape == DICEGPU_QUADRATIC_SF) {
    d.N = 12;
    d.NS = 12;
    const float dl[12] = {0.001f, 0.001f, 1.0e-6f, 1.0e-6f, 1.0e-6f, 1.0f,
                          0.001f, 0.001f, 1.0e-6f, 1.0e-6f, 1.0e-6f, 1.0f};
    for (int i = 0; i < 12; ++i) { d.slot[i] = i; d.deltas[i] = dl[i]; }
    d.has_rot = 0;
  } else {
    d.NS = 6;
    int k = 0;
    d.slot[k++] = 0;
    d.slot[k++] = 1;
    if (p.enable_rotation) d.slot[k++] = 2;
    if (p.enable_normal_strain) { d.slot[k++] = 3; d.slot[k++] = 4; }
    if (p.enable_shear_strain) d.slot[k++] = 5;
    d.N = k;
    for (int i = 0; i < k; ++i) d.deltas[i] = (float)p.robust_delta_theta;
    d.deltas[0] = (float)p.robust_delta_disp;
    d.deltas[1] = (float)p.robust_delta_disp;
    d.has_rot = p.enable_rotation ? 1 : 0;
  }
  d.interp = p.interpolation;
  d.opt = p.optimization;
  d.max_fast = p.max_solver_iterations_fast;
  d.max_robust = p.max_solver_iterations_robust;
  d.fast_tol = (float)p.fast_solver_tolerance;
  d.robust_tol = p.robust_solver_tolerance;
  d.skip_thr = (float)p.skip_solve_gamma_threshold;
  d.skip_all = p.skip_all_solves != 0;
  d.disp_jump = p.disp_jump_tol;
  d.theta_jump = p.theta_jump_tol;
  d.lm_alpha = p.levenberg_marquardt_regularization_factor > 0.0
                   ? (float)p.levenberg_marquardt_regularization_factor : -1.0f;
  d.momentum = (float)p.momentum_factor;
  d.init_gamma_thr = p.initial_gamma_threshold;
  d.final_gamma_thr = p.final_gamma_threshold;
  d.normalize_gamma = p.normalize_gamma_with_active_pixels;
  d.output_beta = p.output_beta;
  d.use_def_grads = p.use_def_gradients;
  d.subset_size = p.subset_size;
  return DICEGPU_OK;
}

extern "C" int dicegpu_default_params(dicegpu_params* p) {
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
  return DICEGPU_OK;
}

// tracking_default_params (DICe_ParameterUtilities.cpp:297-345): the values
// that differ from dice_default_params.
extern "C" int dicegpu_tracking_default_params(dicegpu_params* p) {
  const int rc = dicegpu_default_params(p);
  if (rc) return rc;
  p->correlation_routine = DICEGPU_TRACKING_ROUTINE;
  p->optimization = DICEGPU_SIMPLEX;
  p->enable_rotation = 1;
  p->disp_jump_tol = 8.0;
  p->theta_jump_tol = 0.1;
  p->obstruction_skin_factor = 1.8;
  p->override_force_simplex = 1;
  p->use_subset_evolution = 1;
  return DICEGPU_OK;
}

extern "C" int dicegpu_num_params(const dicegpu_params* p) {
  if (!p) return DICEGPU_ERR_ARG;
  DevParams d;
  const int rc = build_devparams(*p, d);
  return rc ? rc : d.N;
}

extern "C" const char* dicegpu_version(void) { return "dicegpu 1.0 (sm_100a)"; }

extern "C" int dicegpu_create(const dicegpu_params* params, dicegpu_ctx** out) {
  if (!params || !out) return DICEGPU_ERR_ARG;
  *out = nullptr;
  dicegpu_ctx* c = new (std::nothrow) dicegpu_ctx();
  if (!c) return DICEGPU_ERR_NOMEM;
  c->params = *params;
  int rc = build_devparams(*params, c->dp);
  if (rc) { delete c; return rc; }
  if (cudaGetDevice(&c->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&c->smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) != cudaSuccess ||
      cudaMalloc(&c->d_counter, kMaxQueues * sizeof(int)) != cudaSuccess ||
      cudaMalloc(&c->d_status, sizeof(int)) != cudaSuccess ||
      cudaMemset(c->d_status, 0, sizeof(int)) != cudaSuccess) {
    if (c->d_counter) cudaFree(c->d_counter);
    delete c;
    return DICEGPU_ERR_CUDA;
  }
  *out = c;
  return DICEGPU_OK;
}

extern "C" int dicegpu_destroy(dicegpu_ctx* c) {
  if (!c) return DICEGPU_ERR_ARG;
  cudaStreamSynchronize(c->stream);
  cudaFree(c->d_ref); cudaFree(c->d_ref_gx); cudaFree(c->d_ref_gy);
  cudaFree(c->d_def); cudaFree(c->d_def_gx); cudaFree(c->d_def_gy);
  cudaFree(c->d_tmp);
  cudaFree(c->d_def4);
  cudaFree(c->d_fields); cudaFree(c->d_offsets); cudaFree(c->d_px); cudaFree(c->d_py);
  cudaFree(c->d_force); cudaFree(c->d_counter); cudaFree(c->d_status); cudaFree(c->d_passes);
  cudaFree(c->d_unc);
  c->d_shapes.release(); c->d_shape_off.release(); c->d_svx.release(); c->d_svy.release();
  c->d_conformal.release(); c->d_mask_desc.release(); c->d_mask_bits.release();
  c->d_pix_flag.release(); c->d_pix_flag0.release(); c->d_pix_f.release();
  c->d_evo_nact.release(); c->d_evo_nact0.release(); c->d_acc.release(); c->d_ref_saved.release();
  c->d_pix_scratch.release();
  c->d_blk_off.release(); c->d_blk_ids.release(); c->d_neigh.release();
  for (auto& pl : c->plans) { pl.d_wave.release(); pl.d_bwave.release(); }
  c->d_dp_off.release(); c->d_bpoly.release();
  c->d_dv_off.release(); c->d_dvx.release(); c->d_dvy.release();
  c->d_snapshot.release();
  c->d_vsg_cell_off.release(); c->d_vsg_cell_pts.release(); c->d_vsg.release();
  c->d_vsg_pos.release(); c->d_vsg_packed.release(); c->d_vsg_nbr.release();
  if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  delete c;
  return DICEGPU_OK;
}

template <typename T>
static int grow(T** p, size_t* cap, size_t need);

// The uncertainty rows exist while params.compute_uncertainty is set; they
// start at zero for each new set of subsets, like the reference's mesh fields.
static int ensure_uncertainty(dicegpu_ctx* c) {
  if (!c->params.compute_uncertainty || c->n < 1 || c->unc_n == c->n) return DICEGPU_OK;
  const size_t cnt = (size_t)c->n * DICEGPU_UNCERTAINTY_STRIDE;
  int rc = grow(&c->d_unc, &c->unc_cap, cnt);
  if (rc) return rc;
  CK(cudaMemsetAsync(c->d_unc, 0, cnt * sizeof(double), c->stream));
  c->unc_n = c->n;
  return DICEGPU_OK;
}

static int upload_force(dicegpu_ctx* c);

extern "C" int dicegpu_set_params(dicegpu_ctx* c, const dicegpu_params* p) {
  if (!c || !p) return DICEGPU_ERR_ARG;
  DevParams d;
  const int rc = build_devparams(*p, d);
  if (rc) return rc;
  c->params = *p;
  c->dp = d;
  int rc2 = ensure_uncertainty(c);
  if (rc2) return rc2;
  // override_force_simplex decides whether the blocking rule's flags apply
  return (c->n > 0 && !c->h_force_block.empty()) ? upload_force(c) : DICEGPU_OK;
}

extern "C" int dicegpu_get_params(dicegpu_ctx* c, dicegpu_params* p) {
  if (!c || !p) return DICEGPU_ERR_ARG;
  *p = c->params;
  return DICEGPU_OK;
}

extern "C" int dicegpu_set_stream(dicegpu_ctx* c, void* stream) {
  if (!c) return DICEGPU_ERR_ARG;
  c->stream = (cudaStream_t)stream;
  return DICEGPU_OK;
}

static int ensure_images(dicegpu_ctx* c, int w, int h) {
  const size_t npx = (size_t)w * h;
  if (c->has_ref && (c->W != w || c->H != h)) {
    // a new geometry invalidates the previous pair
    c->has_ref = c->has_def = false;
  }
  if (npx > c->img_cap) {
    cudaStreamSynchronize(c->stream);
    float** planes[7] = {&c->d_ref, &c->d_ref_gx, &c->d_ref_gy, &c->d_def, &c->d_def_gx, &c->d_def_gy, &c->d_tmp};
    for (float** pl : planes) { cudaFree(*pl); *pl = nullptr; }
    cudaFree(c->d_def4);
    c->d_def4 = nullptr;
    if (cudaMalloc(&c->d_def4, npx * sizeof(float4)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
    for (int i = 0; i < 6; ++i)
      if (cudaMalloc(planes[i], npx * sizeof(float)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
    if (cudaMalloc(&c->d_tmp, 2 * npx * sizeof(float)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
    c->img_cap = npx;
    c->has_ref = c->has_def = false;
  }
  c->W = w;
  c->H = h;
  return DICEGPU_OK;
}

static int launch_gradients(int w, int h, const float* img, float* gx, float* gy, int method,
                            float* tmp, cudaStream_t st, long long* launches) {
  dim3 blk(256), grd((w + 255) / 256, h);
  if (method == DICEGPU_CONVOLUTION_5_POINT) {
    float* tx = tmp;
    float* ty = tmp + (size_t)w * h;
    gradient_fd_kernel<<<grd, blk, 0, st>>>(w, h, img, tx, ty);
    gradient_smooth_kernel<<<grd, blk, 0, st>>>(w, h, tx, ty, gx, gy);
    if (launches) *launches += 2;
  } else {
    gradient_fd_kernel<<<grd, blk, 0, st>>>(w, h, img, gx, gy);
    if (launches) *launches += 1;
  }
  CK(cudaGetLastError());
  return DICEGPU_OK;
}

// The reference's Gaussian masks are outer products of these 1-D weights
// with every product printed to 9 significant digits (DICe_Image.cpp:54-112);
// rounding the same way gives the identical float tables.
static bool gauss_weights(int M, GaussWeights& g) {
  static const double w5[] = {0.0014, 0.1574, 0.62825};
  static const double w7[] = {0.006, 0.0606, 0.2418, 0.3831};
  static const double w9[] = {0.0007, 0.0108, 0.0748, 0.2384, 0.3505};
  static const double w11[] = {0.0001, 0.0017, 0.0168, 0.087, 0.2328, 0.3231};
  static const double w13[] = {0.0001, 0.0012, 0.0085, 0.038, 0.1109, 0.2108, 0.2611};
  const double* half;
  switch (M) {
    case 5: half = w5; break;
    case 7: half = w7; break;
    case 9: half = w9; break;
    case 11: half = w11; break;
    case 13: half = w13; break;
    default: return false;
  }
  const int R = M / 2;
  double w[13];
  for (int i = 0; i < M; ++i) w[i] = half[i <= R ? i : M - 1 - i];
  for (int i = 0; i < M; ++i)
    for (int j = 0; j < M; ++j) {
      char buf[32];
      std::snprintf(buf, sizeof(buf), "%.8e", w[i] * w[j]);
      g.c[i * M + j] = (float)std::strtod(buf, nullptr);
    }
  return true;
}

static int launch_gauss_filter(int w, int h, int M, const float* in, float* out, cudaStream_t st,
                               long long* launches) {
  GaussWeights g;
  if (!gauss_weights(M, g)) return DICEGPU_ERR_ARG;
  if (w < M || h < M) return DICEGPU_ERR_ARG;
  dim3 blk(kGaussBX, kGaussBY), grd((w + kGaussBX - 1) / kGaussBX, (h + kGaussBY - 1) / kGaussBY);
  gauss_filter_kernel<<<grd, blk, 0, st>>>(w, h, M, g, in, out);
  CK(cudaGetLastError());
  if (launches) *launches += 1;
  return DICEGPU_OK;
}

// Copies the caller's image into dst; with gauss_filter_images the copy goes
// through the filter (raw host pixels are staged in the scratch planes).
static int upload_image(dicegpu_ctx* c, float* dst, const float* src, int on_device) {
  const size_t bytes = (size_t)c->W * c->H * sizeof(float);
  if (c->params.gauss_filter_images) {
    const float* raw = src;
    if (!on_device) {
      CK(cudaMemcpyAsync(c->d_tmp, src, bytes, cudaMemcpyHostToDevice, c->stream));
      raw = c->d_tmp;
    }
    return launch_gauss_filter(c->W, c->H, c->params.gauss_filter_mask_size, raw, dst, c->stream,
                               &c->launches);
  }
  CK(cudaMemcpyAsync(dst, src, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     c->stream));
  return DICEGPU_OK;
}

// 8- and 16-bit pixels become floats of the same value, as the reference's
// image readers store them (DICe_ImageIO.cpp:480-490).
template <typename T>
__global__ void convert_kernel(size_t n, const T* __restrict__ in, float* __restrict__ out) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = (float)in[i];
}

// Integer pixels: the raw bytes are staged in the second scratch plane, the
// conversion writes the first (then the optional filter) or the destination.
static int upload_typed(dicegpu_ctx* c, float* dst, const void* src, int type, int on_device) {
  if (type == DICEGPU_PIXEL_F32) return upload_image(c, dst, (const float*)src, on_device);
  if (type != DICEGPU_PIXEL_U8 && type != DICEGPU_PIXEL_U16) return DICEGPU_ERR_ARG;
  const size_t npx = (size_t)c->W * c->H;
  const size_t esz = type == DICEGPU_PIXEL_U8 ? 1 : 2;
  const void* raw = src;
  if (!on_device) {
    void* stage = (void*)(c->d_tmp + npx);
    CK(cudaMemcpyAsync(stage, src, npx * esz, cudaMemcpyHostToDevice, c->stream));
    raw = stage;
  }
  float* conv = c->params.gauss_filter_images ? c->d_tmp : dst;
  const unsigned blocks = (unsigned)((npx + 255) / 256);
  if (type == DICEGPU_PIXEL_U8)
    convert_kernel<uint8_t><<<blocks, 256, 0, c->stream>>>(npx, (const uint8_t*)raw, conv);
  else
    convert_kernel<uint16_t><<<blocks, 256, 0, c->stream>>>(npx, (const uint16_t*)raw, conv);
  CK(cudaGetLastError());
  c->launches += 1;
  if (c->params.gauss_filter_images)
    return launch_gauss_filter(c->W, c->H, c->params.gauss_filter_mask_size, conv, dst, c->stream,
                               &c->launches);
  return DICEGPU_OK;
}

static int set_ref(dicegpu_ctx* c, int w, int h, const void* pixels, int type, int on_device) {
  if (!c || !pixels || w < 16 || h < 16) return DICEGPU_ERR_ARG;
  int rc = ensure_images(c, w, h);
  if (rc) return rc;
  if ((rc = upload_typed(c, c->d_ref, pixels, type, on_device))) return rc;
  if ((rc = launch_gradients(w, h, c->d_ref, c->d_ref_gx, c->d_ref_gy, c->params.gradient_method,
                             c->d_tmp, c->stream, &c->launches)))
    return rc;
  c->has_ref = true;
  return DICEGPU_OK;
}

static int set_def(dicegpu_ctx* c, int w, int h, const void* pixels, int type, int on_device) {
  if (!c || !pixels) return DICEGPU_ERR_ARG;
  if (!c->has_ref) return DICEGPU_ERR_STATE;
  if (w != c->W || h != c->H) return DICEGPU_ERR_ARG;
  int rc;
  if ((rc = upload_typed(c, c->d_def, pixels, type, on_device))) return rc;
  if (c->params.use_def_gradients) {
    if ((rc = launch_gradients(w, h, c->d_def, c->d_def_gx, c->d_def_gy, c->params.gradient_method,
                               c->d_tmp, c->stream, &c->launches)))
      return rc;
    const size_t npx = (size_t)w * h;
    pack_kernel<<<(unsigned)((npx + 255) / 256), 256, 0, c->stream>>>(npx, c->d_def, c->d_def_gx,
                                                                      c->d_def_gy, c->d_def4);
    CK(cudaGetLastError());
    c->launches += 1;
  }
  c->has_def = true;
  return DICEGPU_OK;
}

extern "C" int dicegpu_set_ref_image(dicegpu_ctx* c, int w, int h, const float* pixels, int on_device) {
  return set_ref(c, w, h, pixels, DICEGPU_PIXEL_F32, on_device);
}
extern "C" int dicegpu_set_def_image(dicegpu_ctx* c, int w, int h, const float* pixels, int on_device) {
  return set_def(c, w, h, pixels, DICEGPU_PIXEL_F32, on_device);
}
extern "C" int dicegpu_set_ref_image_typed(dicegpu_ctx* c, int w, int h, const void* pixels, int pixel_type,
                                           int on_device) {
  return set_ref(c, w, h, pixels, pixel_type, on_device);
}
extern "C" int dicegpu_set_def_image_typed(dicegpu_ctx* c, int w, int h, const void* pixels, int pixel_type,
                                           int on_device) {
  return set_def(c, w, h, pixels, pixel_type, on_device);
}

extern "C" int dicegpu_set_neighbors(dicegpu_ctx* c, const int32_t* neighbor_ids) {
  if (!c || c->n < 1) return DICEGPU_ERR_ARG;
  c->plans[2].valid = c->plans[3].valid = false;   // the plans with neighbours
  if (!neighbor_ids) {
    c->h_neigh.clear();
    return DICEGPU_OK;
  }
  const int n = c->n;
  std::vector<int32_t> nb(neighbor_ids, neighbor_ids + n);
  for (auto& j : nb)
    if (j < 0 || j >= n) j = -1;
  cudaStreamSynchronize(c->stream);
  int rc = c->d_neigh.ensure(n);
  if (rc) return rc;
  CK(cudaMemcpy(c->d_neigh.p, nb.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  c->h_neigh.swap(nb);
  return DICEGPU_OK;
}

extern "C" int dicegpu_set_ref_from_def(dicegpu_ctx* c) {
  if (!c) return DICEGPU_ERR_ARG;
  if (!c->has_ref || !c->has_def) return DICEGPU_ERR_STATE;
  CK(cudaMemcpyAsync(c->d_ref, c->d_def, (size_t)c->W * c->H * sizeof(float), cudaMemcpyDeviceToDevice, c->stream));
  return launch_gradients(c->W, c->H, c->d_ref, c->d_ref_gx, c->d_ref_gy, c->params.gradient_method, c->d_tmp,
                          c->stream, &c->launches);
}

template <typename T>
static int grow(T** p, size_t* cap, size_t need) {
  if (need <= *cap && *p) return DICEGPU_OK;
  cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  if (cudaMalloc(p, std::max<size_t>(need, 1) * sizeof(T)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
  *cap = need;
  return DICEGPU_OK;
}

static void clear_shapes(dicegpu_ctx* c);

extern "C" int dicegpu_set_subsets(dicegpu_ctx* c, int n, const double* fields) {
  if (!c || n < 1 || !fields) return DICEGPU_ERR_ARG;
  cudaStreamSynchronize(c->stream);
  int rc = grow(&c->d_fields, &c->fields_cap, (size_t)n * DICEGPU_FIELD_STRIDE);
  if (rc) return rc;
  rc = grow(&c->d_passes, &c->passes_cap, (size_t)n);
  if (rc) return rc;
  CK(cudaMemcpyAsync(c->d_fields, fields, (size_t)n * DICEGPU_FIELD_STRIDE * sizeof(double),
                     cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (c->n != n) {
    c->use_lists = false;
    c->use_force = false;
    c->h_force_user.clear();
    c->h_skip_user.clear();
    c->h_neigh.clear();
    clear_shapes(c);
  }
  c->vsg_window = 0;
  c->n = n;
  c->frame_index = 0;
  c->unc_n = 0;
  return ensure_uncertainty(c);
}

extern "C" int dicegpu_set_subset_pixels(dicegpu_ctx* c, int n, const int32_t* offsets,
                                         const int32_t* px, const int32_t* py) {
  if (!c || n != c->n || !offsets || !px || !py) return DICEGPU_ERR_ARG;
  if (offsets[0] != 0) return DICEGPU_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (offsets[i + 1] < offsets[i]) return DICEGPU_ERR_ARG;
  const size_t total = (size_t)offsets[n];
  cudaStreamSynchronize(c->stream);
  int rc;
  if ((rc = grow(&c->d_offsets, &c->offs_cap, (size_t)n + 1))) return rc;
  size_t cap2 = c->list_cap;
  if ((rc = grow(&c->d_px, &c->list_cap, total))) return rc;
  if ((rc = grow(&c->d_py, &cap2, total))) return rc;
  c->list_cap = std::min(c->list_cap, cap2);
  CK(cudaMemcpy(c->d_offsets, offsets, (n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (total) {
    CK(cudaMemcpy(c->d_px, px, total * sizeof(int32_t), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->d_py, py, total * sizeof(int32_t), cudaMemcpyHostToDevice));
  }
  c->use_lists = true;
  c->list_npix_max = 0;
  for (int i = 0; i < n; ++i) c->list_npix_max = std::max(c->list_npix_max, offsets[i + 1] - offsets[i]);
  c->has_evo = false;   // explicit lists carry no evolution state
  return DICEGPU_OK;
}

// Bounds of the shape arguments: every coordinate product in the pixel tests
// stays inside int32 and a subset's bounding box stays a bounded walk.
static const int kShapeCoordMax = 1000000;
static const int kShapeExtentMax = 32768;
static const int64_t kShapeAreaMax = (int64_t)1 << 26;

static bool shape_box_host(const dicegpu_shape& s, const int32_t* vx, const int32_t* vy, int64_t& x0,
                           int64_t& x1, int64_t& y0, int64_t& y1) {
  if (s.cx < -kShapeCoordMax || s.cx > kShapeCoordMax || s.cy < -kShapeCoordMax || s.cy > kShapeCoordMax)
    return false;
  if (s.kind == DICEGPU_SHAPE_CIRCLE) {
    if (!(s.radius >= 0.0f && s.radius <= 16384.0f)) return false;
    x0 = (int)((float)s.cx - s.radius - 1.0f); x1 = (int)((float)s.cx + s.radius + 1.0f);
    y0 = (int)((float)s.cy - s.radius - 1.0f); y1 = (int)((float)s.cy + s.radius + 1.0f);
  } else if (s.kind == DICEGPU_SHAPE_RECTANGLE) {
    if (s.width < 0 || s.width > kShapeExtentMax || s.height < 0 || s.height > kShapeExtentMax) return false;
    x0 = s.cx - s.width / 2; x1 = x0 + s.width - 1;
    y0 = s.cy - s.height / 2; y1 = y0 + s.height - 1;
  } else if (s.kind == DICEGPU_SHAPE_POLYGON) {
    if (!vx || !vy || s.vertex_count < 3 || s.vertex_count > 4096 || s.vertex_offset < 0) return false;
    x0 = y0 = INT64_MAX; x1 = y1 = INT64_MIN;
    for (int k = 0; k < s.vertex_count; ++k) {
      const int64_t x = vx[s.vertex_offset + k], y = vy[s.vertex_offset + k];
      if (x < -kShapeCoordMax || x > kShapeCoordMax || y < -kShapeCoordMax || y > kShapeCoordMax) return false;
      x0 = std::min(x0, x); x1 = std::max(x1, x); y0 = std::min(y0, y); y1 = std::max(y1, y);
    }
  } else {
    return false;
  }
  return true;
}

// The device force-simplex flags: the caller's, and those of blocked and
// blocking subsets unless params.override_force_simplex.
static int upload_force(dicegpu_ctx* c) {
  const int n = c->n;
  const bool user = (int)c->h_force_user.size() == n;
  const bool block = (int)c->h_force_block.size() == n && !c->params.override_force_simplex;
  const bool skip = (int)c->h_skip_user.size() == n;
  if (!user && !block && !skip) {
    c->use_force = false;
    return DICEGPU_OK;
  }
  // per subset: bit 0 force the simplex, bit 1 skip the solve
  std::vector<uint8_t> f(n, 0);
  for (int i = 0; i < n; ++i)
    f[i] = (uint8_t)(((user && c->h_force_user[i]) || (block && c->h_force_block[i]) ? 1 : 0) |
                     (skip && c->h_skip_user[i] ? 2 : 0));
  cudaStreamSynchronize(c->stream);
  int rc = grow(&c->d_force, &c->force_cap, (size_t)n);
  if (rc) return rc;
  CK(cudaMemcpy(c->d_force, f.data(), n, cudaMemcpyHostToDevice));
  c->use_force = true;
  return DICEGPU_OK;
}

static void clear_shapes(dicegpu_ctx* c) {
  c->h_shapes.clear(); c->h_shape_off.clear(); c->h_svx.clear(); c->h_svy.clear();
  c->h_conformal.clear(); c->h_mask_desc.clear();
  c->use_masks = false;
  c->has_evo = false;
  c->has_blocking = false;
  c->h_blk_off.clear(); c->h_blk_ids.clear();
  c->blocking_desc_ready = false;
  for (auto& pl : c->plans) pl.valid = false;
  c->n_blocked = 0;
  c->h_force_block.clear();
}

extern "C" int dicegpu_set_subset_shapes(dicegpu_ctx* c, int n_shapes, const dicegpu_shape* shapes,
                                         const int32_t* vx, const int32_t* vy) {
  if (!c || c->n < 1 || n_shapes < 1 || !shapes) return DICEGPU_ERR_ARG;
  const int n = c->n;
  // validate, bound every subset's boxes, and group the shapes by subset
  int64_t n_vertices = 0;
  std::vector<int64_t> bx0(n, INT64_MAX), bx1(n, INT64_MIN), by0(n, INT64_MAX), by1(n, INT64_MIN);
  std::vector<int64_t> ox0(n, INT64_MAX), ox1(n, INT64_MIN), oy0(n, INT64_MAX), oy1(n, INT64_MIN);
  std::vector<int32_t> shape_off(n + 1, 0);
  for (int k = 0; k < n_shapes; ++k) {
    const dicegpu_shape& s = shapes[k];
    if (s.subset < 0 || s.subset >= n || s.role < DICEGPU_ROLE_BOUNDARY || s.role > DICEGPU_ROLE_OBSTRUCTED)
      return DICEGPU_ERR_ARG;
    int64_t x0, x1, y0, y1;
    if (!shape_box_host(s, vx, vy, x0, x1, y0, y1)) return DICEGPU_ERR_ARG;
    if (s.kind == DICEGPU_SHAPE_POLYGON)
      n_vertices = std::max<int64_t>(n_vertices, (int64_t)s.vertex_offset + s.vertex_count);
    if (s.role == DICEGPU_ROLE_BOUNDARY) {
      bx0[s.subset] = std::min(bx0[s.subset], x0); bx1[s.subset] = std::max(bx1[s.subset], x1);
      by0[s.subset] = std::min(by0[s.subset], y0); by1[s.subset] = std::max(by1[s.subset], y1);
    } else if (s.role == DICEGPU_ROLE_OBSTRUCTED) {
      ox0[s.subset] = std::min(ox0[s.subset], x0); ox1[s.subset] = std::max(ox1[s.subset], x1);
      oy0[s.subset] = std::min(oy0[s.subset], y0); oy1[s.subset] = std::max(oy1[s.subset], y1);
    }
    ++shape_off[s.subset + 1];
  }
  auto box_ok = [](int64_t a0, int64_t a1, int64_t b0, int64_t b1) {
    if (a1 < a0) return true;   // none
    const int64_t w = a1 - a0 + 1, h = b1 - b0 + 1;
    return w <= kShapeExtentMax && h <= kShapeExtentMax && w * h <= kShapeAreaMax;
  };
  for (int i = 0; i < n; ++i)
    if (!box_ok(bx0[i], bx1[i], by0[i], by1[i]) || !box_ok(ox0[i], ox1[i], oy0[i], oy1[i]))
      return DICEGPU_ERR_ARG;
  for (int i = 0; i < n; ++i) shape_off[i + 1] += shape_off[i];
  std::vector<dicegpu_shape> grouped(n_shapes);
  {
    std::vector<int32_t> fill(shape_off.begin(), shape_off.end() - 1);
    for (int k = 0; k < n_shapes; ++k) grouped[fill[shapes[k].subset]++] = shapes[k];
  }
  // obstruction boxes and word offsets
  std::vector<int32_t> desc((size_t)n * DG_MASK_DESC, 0), obst_list;
  int64_t obst_words = 0;
  for (int i = 0; i < n; ++i) {
    if (ox1[i] < ox0[i]) continue;
    int32_t* d = &desc[(size_t)i * DG_MASK_DESC];
    d[0] = (int32_t)ox0[i]; d[1] = (int32_t)oy0[i];
    d[2] = (int32_t)(ox1[i] - ox0[i] + 1); d[3] = (int32_t)(oy1[i] - oy0[i] + 1);
    d[4] = (int32_t)obst_words;
    obst_words += ((int64_t)d[2] * d[3] + 31) / 32;
    obst_list.push_back(i);
  }
  if (obst_words > ((int64_t)1 << 31)) return DICEGPU_ERR_ARG;
  std::vector<uint8_t> conformal(n, 0);
  for (int i = 0; i < n; ++i) conformal[i] = bx1[i] >= bx0[i];
  // subset evolution keeps the excluded pixels of conformal subsets with
  // excluded shapes in their lists (the reference's static tracking
  // objectives carry them, inactive, from frame to frame)
  const bool evolution = c->params.use_subset_evolution && c->params.correlation_routine == DICEGPU_TRACKING_ROUTINE;
  bool any_evo = false;
  if (evolution)
    for (int k = 0; k < n_shapes; ++k) {
      const dicegpu_shape& s = grouped[k];
      if (s.role == DICEGPU_ROLE_EXCLUDED && conformal[s.subset]) {
        desc[(size_t)s.subset * DG_MASK_DESC + DG_DESC_EVOLVE] = 1;
        any_evo = true;
      }
    }
  cudaStreamSynchronize(c->stream);
  const size_t nv = (size_t)std::max<int64_t>(n_vertices, 1);
  int rc;
  if ((rc = c->d_shapes.ensure(n_shapes)) || (rc = c->d_shape_off.ensure(n + 1)) || (rc = c->d_svx.ensure(nv)) ||
      (rc = c->d_svy.ensure(nv)) || (rc = c->d_conformal.ensure(n)))
    return rc;
  int32_t* d_counts = nullptr;
  if (cudaMalloc(&d_counts, n * sizeof(int32_t)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
  std::vector<int32_t> counts(n), offsets(n + 1, 0);
  if (any_evo && ((rc = c->d_evo_nact0.ensure(n)) || (rc = c->d_evo_nact.ensure(n)))) {
    cudaFree(d_counts);
    return rc;
  }
  RasterArgs ra{c->d_shapes.p, c->d_shape_off.p, c->d_svx.p, c->d_svy.p, n, d_counts, nullptr, nullptr, nullptr,
                c->d_fields, c->params.subset_size >= 1 ? c->params.subset_size / 2 : -1,
                any_evo ? 1 : 0, nullptr, any_evo ? c->d_evo_nact0.p : nullptr};
  const unsigned blocks = (unsigned)std::min<int64_t>(((int64_t)n * 32 + 255) / 256, (int64_t)c->num_sms * 8);
  cudaError_t e = cudaMemcpy(c->d_shapes.p, grouped.data(), n_shapes * sizeof(dicegpu_shape), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(c->d_shape_off.p, shape_off.data(), (n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && n_vertices) {
    e = cudaMemcpy(c->d_svx.p, vx, n_vertices * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(c->d_svy.p, vy, n_vertices * sizeof(int32_t), cudaMemcpyHostToDevice);
  }
  if (e == cudaSuccess) e = cudaMemcpy(c->d_conformal.p, conformal.data(), n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    raster_kernel<false><<<blocks, 256, 0, c->stream>>>(ra);
    ++c->launches;
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(counts.data(), d_counts, n * sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  cudaFree(d_counts);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return DICEGPU_ERR_CUDA;
  }
  for (int i = 0; i < n; ++i) {
    offsets[i + 1] = offsets[i] + counts[i];
    if (offsets[i + 1] < offsets[i]) return DICEGPU_ERR_ARG;   // > 2^31 pixels
  }
  const size_t total = (size_t)offsets[n];
  if ((rc = grow(&c->d_offsets, &c->offs_cap, (size_t)n + 1))) return rc;
  size_t cap2 = c->list_cap;
  if ((rc = grow(&c->d_px, &c->list_cap, total)) || (rc = grow(&c->d_py, &cap2, total))) return rc;
  c->list_cap = std::min(c->list_cap, cap2);
  CK(cudaMemcpy(c->d_offsets, offsets.data(), (n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (any_evo) {
    const size_t t1 = std::max<size_t>(total, 1);
    if ((rc = c->d_pix_flag0.ensure(t1)) || (rc = c->d_pix_flag.ensure(t1)) || (rc = c->d_pix_f.ensure(t1)))
      return rc;
  }
  ra.offsets = c->d_offsets;
  ra.px = c->d_px;
  ra.py = c->d_py;
  ra.active = nullptr;
  ra.flags = any_evo ? c->d_pix_flag0.p : nullptr;
  raster_kernel<true><<<blocks, 256, 0, c->stream>>>(ra);
  ++c->launches;
  CK(cudaGetLastError());
  // obstruction bitmaps
  clear_shapes(c);
  if (!obst_list.empty() || any_evo) {
    if ((rc = c->d_mask_desc.ensure(desc.size()))) return rc;
    CK(cudaMemcpyAsync(c->d_mask_desc.p, desc.data(), desc.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                       c->stream));
    c->use_masks = true;
  }
  if (any_evo) {
    // the evolution state of a fresh sequence
    c->evo_total = std::max<size_t>(total, 1);
    CK(cudaMemcpyAsync(c->d_pix_flag.p, c->d_pix_flag0.p, c->evo_total, cudaMemcpyDeviceToDevice, c->stream));
    CK(cudaMemsetAsync(c->d_pix_f.p, 0, c->evo_total * sizeof(float), c->stream));
    CK(cudaMemcpyAsync(c->d_evo_nact.p, c->d_evo_nact0.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                       c->stream));
    c->has_evo = true;
  }
  if (!obst_list.empty()) {
    if ((rc = c->d_mask_bits.ensure((size_t)obst_words))) return rc;
    int32_t* d_list = nullptr;
    if (cudaMalloc(&d_list, obst_list.size() * sizeof(int32_t)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
    e = cudaMemsetAsync(c->d_mask_bits.p, 0, (size_t)obst_words * sizeof(uint32_t), c->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_list, obst_list.data(), obst_list.size() * sizeof(int32_t), cudaMemcpyHostToDevice,
                          c->stream);
    if (e == cudaSuccess) {
      ObstArgs oa{c->d_shapes.p, c->d_shape_off.p, c->d_svx.p, c->d_svy.p, d_list, (int)obst_list.size(),
                  c->d_mask_desc.p, c->d_mask_bits.p};
      const unsigned ob = (unsigned)std::min<int64_t>(((int64_t)obst_list.size() * 32 + 255) / 256,
                                                      (int64_t)c->num_sms * 8);
      obstruction_kernel<<<ob, 256, 0, c->stream>>>(oa);
      ++c->launches;
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(d_list);
    if (e != cudaSuccess) {
    cudaGetLastError();
    return DICEGPU_ERR_CUDA;
  }
    c->use_masks = true;
  }
  c->h_shapes.swap(grouped);
  c->h_shape_off.swap(shape_off);
  if (n_vertices) {
    c->h_svx.assign(vx, vx + n_vertices);
    c->h_svy.assign(vy, vy + n_vertices);
  }
  c->h_conformal.swap(conformal);
  c->h_mask_desc.swap(desc);
  CK(cudaStreamSynchronize(c->stream));
  c->use_lists = true;
  c->list_npix_max = 0;
  for (int i = 0; i < n; ++i) c->list_npix_max = std::max(c->list_npix_max, counts[i]);
  return upload_force(c);
}

extern "C" int dicegpu_set_blocking(dicegpu_ctx* c, const int32_t* offsets, const int32_t* ids) {
  if (!c || c->n < 1) return DICEGPU_ERR_ARG;
  const int n = c->n;
  cudaStreamSynchronize(c->stream);
  if (!offsets) {
    c->has_blocking = false;
    c->h_force_block.clear();
    c->n_blocked = 0;
    for (auto& pl : c->plans) pl.valid = false;
    if (!c->h_mask_desc.empty()) {
      bool any = false;
      for (int i = 0; i < n; ++i) {
        int32_t* d = &c->h_mask_desc[(size_t)i * DG_MASK_DESC];
        d[5] = d[6] = 0;
        any = any || d[2] > 0 || d[DG_DESC_EVOLVE] != 0;
      }
      // the device descriptors exist once an obstruction or a tracking frame needed them
      if (c->d_mask_desc.p && c->d_mask_desc.cap >= c->h_mask_desc.size())
        CK(cudaMemcpy(c->d_mask_desc.p, c->h_mask_desc.data(), c->h_mask_desc.size() * sizeof(int32_t),
                      cudaMemcpyHostToDevice));
      c->use_masks = any;
      c->blocking_desc_ready = false;
    }
    return upload_force(c);
  }
  if (offsets[0] != 0 || (offsets[n] > 0 && !ids)) return DICEGPU_ERR_ARG;
  for (int i = 0; i < n; ++i)
    if (offsets[i + 1] < offsets[i]) return DICEGPU_ERR_ARG;
  for (int k = 0; k < offsets[n]; ++k)
    if (ids[k] < 0 || ids[k] >= n) return DICEGPU_ERR_ARG;
  const bool have_shapes = (int)c->h_conformal.size() == n;
  // deformed vertices and polygon-table slots per blocked subset
  std::vector<int32_t> dv_off, dp_off(n, 0);
  std::vector<uint8_t> force(n, 0), has_polys(n, 0);
  int64_t dv_total = 0, dp_total = 0;
  int n_blocked = 0;
  for (int i = 0; i < n; ++i) {
    if (offsets[i + 1] > offsets[i]) force[i] = 1;   // blocked
    int polys = 0;
    int64_t verts = 0;
    for (int k = offsets[i]; k < offsets[i + 1]; ++k) {
      const int j = ids[k];
      force[j] = 1;   // blocking
      if (!have_shapes || !c->h_conformal[j]) continue;
      for (int m = c->h_shape_off[j]; m < c->h_shape_off[j + 1]; ++m) {
        const dicegpu_shape& s = c->h_shapes[m];
        if (s.role != DICEGPU_ROLE_BOUNDARY) continue;
        if (s.kind == DICEGPU_SHAPE_CIRCLE) return DICEGPU_ERR_UNSUPPORTED;
        ++polys;
        verts += s.kind == DICEGPU_SHAPE_RECTANGLE ? 4 : s.vertex_count;
      }
    }
    if (polys > DG_MAX_BLOCK_POLYS) return DICEGPU_ERR_UNSUPPORTED;
    dv_off.push_back((int32_t)dv_total);
    dp_off[i] = (int32_t)dp_total;
    if (polys > 0) {
      has_polys[i] = 1;
      ++n_blocked;
      dv_total += verts;
      dp_total += polys;
    }
  }
  if (dv_total > ((int64_t)1 << 30) || dp_total > ((int64_t)1 << 26)) return DICEGPU_ERR_ARG;
  int rc;
  if ((rc = c->d_blk_off.ensure(n + 1)) || (rc = c->d_blk_ids.ensure(std::max(offsets[n], 1))) ||
      (rc = c->d_dv_off.ensure(n)) || (rc = c->d_dvx.ensure((size_t)std::max<int64_t>(dv_total, 1))) ||
      (rc = c->d_dvy.ensure((size_t)std::max<int64_t>(dv_total, 1))) || (rc = c->d_dp_off.ensure(n)) ||
      (rc = c->d_bpoly.ensure(6 * (size_t)std::max<int64_t>(dp_total, 1))) ||
      (rc = c->d_snapshot.ensure((size_t)n * DICEGPU_FIELD_STRIDE)))
    return rc;
  CK(cudaMemcpy(c->d_blk_off.p, offsets, (n + 1) * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (offsets[n]) CK(cudaMemcpy(c->d_blk_ids.p, ids, offsets[n] * sizeof(int32_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_dv_off.p, dv_off.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_dp_off.p, dp_off.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  c->h_blk_off.assign(offsets, offsets + n + 1);
  c->h_blk_ids.assign(ids, ids + offsets[n]);
  c->h_has_polys.swap(has_polys);
  for (auto& pl : c->plans) pl.valid = false;
  c->n_blocked = n_blocked;
  c->blocking_desc_ready = false;   // descriptors uploaded at the next tracking frame
  c->h_force_block.swap(force);
  c->has_blocking = true;
  if (c->h_mask_desc.empty()) c->h_mask_desc.assign((size_t)n * DG_MASK_DESC, 0);
  return upload_force(c);
}

// Puts the mask descriptors on the device for the tracking waves (the
// blocked-polygon counts start at zero; blocked_kernel fills them).
static int ensure_blocking_desc(dicegpu_ctx* c) {
  if (c->blocking_desc_ready) return DICEGPU_OK;
  cudaStreamSynchronize(c->stream);
  int rc;
  if ((rc = c->d_mask_desc.ensure(c->h_mask_desc.size()))) return rc;
  for (int i = 0; i < c->n; ++i) {
    int32_t* d = &c->h_mask_desc[(size_t)i * DG_MASK_DESC];
    d[5] = d[6] = 0;
  }
  CK(cudaMemcpy(c->d_mask_desc.p, c->h_mask_desc.data(), c->h_mask_desc.size() * sizeof(int32_t),
                cudaMemcpyHostToDevice));
  c->blocking_desc_ready = true;
  c->use_masks = true;
  return DICEGPU_OK;
}

// ---------------------------------------------------------------------------
// VSG strain (VSG_Strain_Post_Processor)
// ---------------------------------------------------------------------------
// The uniform grid of the subset centres for a window: cell size >= the
// search radius + 1 px, so the 3 x 3 cells around a centre hold every
// neighbour even when a centre sits on a cell edge.
static int build_vsg_grid(dicegpu_ctx* c, int window) {
  const int n = c->n;
  std::vector<double> rows((size_t)n * DICEGPU_FIELD_STRIDE);
  CK(cudaMemcpyAsync(rows.data(), c->d_fields, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  // radius of the reference's neighbourhood search (initialize_neighborhood)
  const float rad = (float)((float)window / 2.0);
  const float r2 = rad * rad + 1.0e-5f;
  float x0 = 0.0f, y0 = 0.0f, x1 = 0.0f, y1 = 0.0f;
  for (int i = 0; i < n; ++i) {
    const float x = (float)rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X];
    const float y = (float)rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y];
    if (!std::isfinite(x) || !std::isfinite(y)) return DICEGPU_ERR_ARG;
    if (i == 0 || x < x0) x0 = x;
    if (i == 0 || y < y0) y0 = y;
    if (i == 0 || x > x1) x1 = x;
    if (i == 0 || y > y1) y1 = y;
  }
  float cell = std::ceil(std::sqrt(r2)) + 1.0f;
  // at most ~4 cells per subset: sparse centres over a wide field get wider cells
  while (((double)(x1 - x0) / cell + 1.0) * ((double)(y1 - y0) / cell + 1.0) > 4.0 * n + 16.0) cell *= 2.0f;
  const int ncx = (int)std::floor((x1 - x0) / cell) + 1, ncy = (int)std::floor((y1 - y0) / cell) + 1;
  std::vector<int32_t> off((size_t)ncx * ncy + 1, 0), pts(n), cell_of(n);
  for (int i = 0; i < n; ++i) {
    const float x = (float)rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X];
    const float y = (float)rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y];
    const int gx = std::min(std::max((int)std::floor((x - x0) / cell), 0), ncx - 1);
    const int gy = std::min(std::max((int)std::floor((y - y0) / cell), 0), ncy - 1);
    cell_of[i] = gy * ncx + gx;
    ++off[cell_of[i] + 1];
  }
  for (size_t k = 0; k + 1 < off.size(); ++k) off[k + 1] += off[k];
  std::vector<int32_t> pos(n);
  {
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int i = 0; i < n; ++i) {
      pos[i] = fill[cell_of[i]]++;
      pts[pos[i]] = i;
    }
  }
  int rc;
  if ((rc = c->d_vsg_cell_off.ensure(off.size())) || (rc = c->d_vsg_cell_pts.ensure(n)) ||
      (rc = c->d_vsg_pos.ensure(n)) || (rc = c->d_vsg_packed.ensure(n)))
    return rc;
  CK(cudaMemcpy(c->d_vsg_cell_off.p, off.data(), off.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_vsg_cell_pts.p, pts.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->d_vsg_pos.p, pos.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  c->h_vsg_coords.resize(2 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    c->h_vsg_coords[2 * i] = rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X];
    c->h_vsg_coords[2 * i + 1] = rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y];
  }
  c->vsg_ncx = ncx;
  c->vsg_ncy = ncy;
  c->vsg_x0 = x0;
  c->vsg_y0 = y0;
  c->vsg_cell = cell;
  c->vsg_r2 = r2;
  c->vsg_window = window;
  return DICEGPU_OK;
}

// The k nearest subsets of every subset (a negative VSG window), valid or
// not, in ascending float squared distance (query minus point, as the
// kd-tree's L2 adaptor forms it), ties by index.  Candidates come from a
// uniform grid of about k / 4 subsets per cell, searched in growing squares
// of cells until the k-th distance is below the square's inner radius, so
// no closer point lies outside it.
static int build_vsg_knn(dicegpu_ctx* c, int k) {
  const int n = c->n;
  if (k > n) return DICEGPU_ERR_ARG;
  std::vector<double> rows((size_t)n * DICEGPU_FIELD_STRIDE);
  CK(cudaMemcpyAsync(rows.data(), c->d_fields, rows.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  std::vector<float> px(n), py(n);
  float x0 = 0.0f, y0 = 0.0f, x1 = 0.0f, y1 = 0.0f;
  for (int i = 0; i < n; ++i) {
    px[i] = (float)rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X];
    py[i] = (float)rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y];
    if (!std::isfinite(px[i]) || !std::isfinite(py[i])) return DICEGPU_ERR_ARG;
    if (i == 0 || px[i] < x0) x0 = px[i];
    if (i == 0 || py[i] < y0) y0 = py[i];
    if (i == 0 || px[i] > x1) x1 = px[i];
    if (i == 0 || py[i] > y1) y1 = py[i];
  }
  const double area = std::max(1.0, ((double)x1 - x0 + 1.0) * ((double)y1 - y0 + 1.0));
  const double cell = std::max(1.0, std::sqrt(area / n * std::max(k, 4) / 4.0));
  const int ncx = (int)std::floor((x1 - x0) / cell) + 1, ncy = (int)std::floor((y1 - y0) / cell) + 1;
  std::vector<int32_t> off((size_t)ncx * ncy + 1, 0), pts(n), cell_of(n);
  for (int i = 0; i < n; ++i) {
    const int gx = std::min((int)std::floor((px[i] - x0) / cell), ncx - 1);
    const int gy = std::min((int)std::floor((py[i] - y0) / cell), ncy - 1);
    cell_of[i] = gy * ncx + gx;
    ++off[cell_of[i] + 1];
  }
  for (size_t q = 0; q + 1 < off.size(); ++q) off[q + 1] += off[q];
  {
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (int i = 0; i < n; ++i) pts[fill[cell_of[i]]++] = i;
  }
  std::vector<int32_t> nbr((size_t)n * k);
  std::vector<std::pair<float, int32_t>> cand;
  for (int i = 0; i < n; ++i) {
    const int gx = cell_of[i] % ncx, gy = cell_of[i] / ncx;
    for (int R = 1;; ++R) {
      cand.clear();
      for (int cy = std::max(gy - R, 0); cy <= std::min(gy + R, ncy - 1); ++cy) {
        const int q0 = off[(size_t)cy * ncx + std::max(gx - R, 0)];
        const int q1 = off[(size_t)cy * ncx + std::min(gx + R, ncx - 1) + 1];
        for (int q = q0; q < q1; ++q) {
          const int j = pts[q];
          const float dx = px[i] - px[j], dy = py[i] - py[j];
          cand.push_back(std::make_pair(dx * dx + dy * dy, j));
        }
      }
      const bool all = gx - R <= 0 && gy - R <= 0 && gx + R >= ncx - 1 && gy + R >= ncy - 1;
      if ((int)cand.size() < k && !all) continue;
      std::partial_sort(cand.begin(), cand.begin() + k, cand.end());
      // a point outside the square is at least R cells away in x or y
      const double inner = R * cell;
      if (all || (double)cand[k - 1].first < inner * inner * (1.0 - 1e-6)) break;
    }
    for (int q = 0; q < k; ++q) nbr[(size_t)i * k + q] = cand[q].second;
  }
  int rc;
  if ((rc = c->d_vsg_nbr.ensure(nbr.size()))) return rc;
  CK(cudaMemcpy(c->d_vsg_nbr.p, nbr.data(), nbr.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  c->h_vsg_coords.resize(2 * (size_t)n);
  for (int i = 0; i < n; ++i) {
    c->h_vsg_coords[2 * i] = rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X];
    c->h_vsg_coords[2 * i + 1] = rows[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y];
  }
  c->vsg_window = -k;
  return DICEGPU_OK;
}

extern "C" int dicegpu_vsg_strain(dicegpu_ctx* c, int window_size, double* out, int on_device) {
  if (!c || c->n < 1 || window_size == 0) return DICEGPU_ERR_ARG;
  int rc;
  if (window_size < 0) {
    if (c->vsg_window != window_size && (rc = build_vsg_knn(c, -window_size))) return rc;
    if ((rc = c->d_vsg.ensure((size_t)c->n * DICEGPU_VSG_STRIDE))) return rc;
    VsgKnnArgs ka{c->d_fields, c->n, -window_size, c->d_vsg_nbr.p, c->d_vsg.p};
    const unsigned blocks = (unsigned)std::min<int64_t>(((int64_t)c->n + 255) / 256, (int64_t)c->num_sms * 8);
    vsg_knn_kernel<<<blocks, 256, 0, c->stream>>>(ka);
    CK(cudaGetLastError());
    c->launches += 1;
    if (out)
      CK(cudaMemcpyAsync(out, c->d_vsg.p, (size_t)c->n * DICEGPU_VSG_STRIDE * sizeof(double),
                         on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
    if (out && !on_device) CK(cudaStreamSynchronize(c->stream));
    return DICEGPU_OK;
  }
  if (c->vsg_window != window_size && (rc = build_vsg_grid(c, window_size))) return rc;
  if ((rc = c->d_vsg.ensure((size_t)c->n * DICEGPU_VSG_STRIDE))) return rc;
  VsgArgs va{c->d_fields, c->n, c->d_vsg_cell_off.p, c->d_vsg_cell_pts.p, c->d_vsg_pos.p, c->d_vsg_packed.p,
             c->vsg_ncx, c->vsg_ncy, c->vsg_x0, c->vsg_y0, c->vsg_cell, c->vsg_r2, c->d_vsg.p};
  const unsigned pblocks = (unsigned)std::min<int64_t>(((int64_t)c->n + 255) / 256, (int64_t)c->num_sms * 8);
  vsg_pack_kernel<<<pblocks, 256, 0, c->stream>>>(va);
  // one warp per 32 subsets
  const unsigned blocks = (unsigned)std::min<int64_t>(((int64_t)c->n + 255) / 256, (int64_t)c->num_sms * 16);
  vsg_kernel<<<blocks, 256, 0, c->stream>>>(va);
  CK(cudaGetLastError());
  c->launches += 2;
  if (out)
    CK(cudaMemcpyAsync(out, c->d_vsg.p, (size_t)c->n * DICEGPU_VSG_STRIDE * sizeof(double),
                       on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  if (out && !on_device) CK(cudaStreamSynchronize(c->stream));
  return DICEGPU_OK;
}

extern "C" int dicegpu_get_subset_pixels(dicegpu_ctx* c, int32_t* offsets, int32_t* px, int32_t* py) {
  if (!c || !offsets || !c->use_lists || c->n < 1) return DICEGPU_ERR_ARG;
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaMemcpy(offsets, c->d_offsets, (c->n + 1) * sizeof(int32_t), cudaMemcpyDeviceToHost));
  const size_t total = (size_t)offsets[c->n];
  if (px && total) CK(cudaMemcpy(px, c->d_px, total * sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (py && total) CK(cudaMemcpy(py, c->d_py, total * sizeof(int32_t), cudaMemcpyDeviceToHost));
  return DICEGPU_OK;
}

extern "C" int dicegpu_get_subset_pixel_state(dicegpu_ctx* c, uint8_t* state, float* ref_values) {
  if (!c || (!state && !ref_values)) return DICEGPU_ERR_ARG;
  if (!c->has_evo) return DICEGPU_ERR_STATE;
  CK(cudaStreamSynchronize(c->stream));
  int32_t last = 0;
  CK(cudaMemcpy(&last, c->d_offsets + c->n, sizeof(int32_t), cudaMemcpyDeviceToHost));
  if (last > 0 && state) CK(cudaMemcpy(state, c->d_pix_flag.p, (size_t)last, cudaMemcpyDeviceToHost));
  if (last > 0 && ref_values)
    CK(cudaMemcpy(ref_values, c->d_pix_f.p, (size_t)last * sizeof(float), cudaMemcpyDeviceToHost));
  return DICEGPU_OK;
}

extern "C" int dicegpu_set_skip_solve(dicegpu_ctx* c, int n, const uint8_t* flags) {
  if (!c) return DICEGPU_ERR_ARG;
  if (!flags) {
    c->h_skip_user.clear();
    return upload_force(c);
  }
  if (n != c->n) return DICEGPU_ERR_ARG;
  c->h_skip_user.assign(flags, flags + n);
  return upload_force(c);
}

extern "C" int dicegpu_skip_solve_frame(const int32_t* frame_ids, int count, int frame) {
  if (count < 0 || (count > 0 && !frame_ids)) return DICEGPU_ERR_ARG;
  if (count == 0) return 1;
  int index = count;
  for (int i = 0; i < count; ++i)
    if (frame < frame_ids[i]) {
      index = i;
      break;
    }
  return index % 2 == 0 ? 0 : 1;
}

extern "C" int dicegpu_set_force_simplex(dicegpu_ctx* c, int n, const uint8_t* flags) {
  if (!c) return DICEGPU_ERR_ARG;
  if (!flags) {
    c->h_force_user.clear();
    return upload_force(c);
  }
  if (n != c->n) return DICEGPU_ERR_ARG;
  c->h_force_user.assign(flags, flags + n);
  return upload_force(c);
}

extern "C" int dicegpu_get_fields(dicegpu_ctx* c, double* out) {
  if (!c || !out || c->n < 1) return DICEGPU_ERR_ARG;
  CK(cudaMemcpyAsync(out, c->d_fields, (size_t)c->n * DICEGPU_FIELD_STRIDE * sizeof(double),
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DICEGPU_OK;
}

extern "C" int dicegpu_num_subsets(dicegpu_ctx* c, int* n) {
  if (!c || !n) return DICEGPU_ERR_ARG;
  *n = c->n;
  return DICEGPU_OK;
}

extern "C" int dicegpu_get_uncertainty(dicegpu_ctx* c, double* out) {
  if (!c || !out || c->n < 1) return DICEGPU_ERR_ARG;
  if (!c->params.compute_uncertainty || c->unc_n != c->n) return DICEGPU_ERR_STATE;
  CK(cudaMemcpyAsync(out, c->d_unc, (size_t)c->n * DICEGPU_UNCERTAINTY_STRIDE * sizeof(double),
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DICEGPU_OK;
}

extern "C" int dicegpu_load_fields(dicegpu_ctx* c, const double* src, int on_device) {
  if (!c || !src || c->n < 1) return DICEGPU_ERR_ARG;
  CK(cudaMemcpyAsync(c->d_fields, src, (size_t)c->n * DICEGPU_FIELD_STRIDE * sizeof(double),
                     on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
  c->frame_index = 0;
  // the VSG neighbour grid stays valid when host rows keep its coordinates
  bool same = !on_device && c->vsg_window != 0 && c->h_vsg_coords.size() == 2 * (size_t)c->n;
  for (int i = 0; same && i < c->n; ++i)
    same = src[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_X] == c->h_vsg_coords[2 * i] &&
           src[(size_t)i * DICEGPU_FIELD_STRIDE + DICEGPU_F_COORD_Y] == c->h_vsg_coords[2 * i + 1];
  if (!same) c->vsg_window = 0;
  return DICEGPU_OK;
}

extern "C" int dicegpu_store_fields(dicegpu_ctx* c, double* dst, int on_device) {
  if (!c || !dst || c->n < 1) return DICEGPU_ERR_ARG;
  CK(cudaMemcpyAsync(dst, c->d_fields, (size_t)c->n * DICEGPU_FIELD_STRIDE * sizeof(double),
                     on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, c->stream));
  return DICEGPU_OK;
}

extern "C" int dicegpu_fields_device_ptr(dicegpu_ctx* c, double** dptr) {
  if (!c || !dptr) return DICEGPU_ERR_ARG;
  *dptr = c->d_fields;
  return DICEGPU_OK;
}

// the largest pixel count of a subset of the context (squares: side^2)
static int npix_max(const dicegpu_ctx* c) {
  if (c->use_lists) return std::max(c->list_npix_max, 1);
  const int side = 2 * (c->params.subset_size / 2) + 1;
  return side * side;
}

// dynamic shared memory of a frame CTA of `warps` warps: the control block,
// per-warp sums, simplex state and staging (`fixed`), and the per-pixel
// arrays (`pix`)
static void frame_smem_bytes(const dicegpu_ctx* c, int warps, size_t* fixed, size_t* pix) {
  const int cap = pix_cap(npix_max(c));
  if (c->dp.shape == DICEGPU_QUADRATIC_SF) {
    *fixed = SmemPlan<DICEGPU_QUADRATIC_SF>::pix(warps);
    *pix = SmemPlan<DICEGPU_QUADRATIC_SF>::pix_bytes(cap);
  } else {
    *fixed = SmemPlan<DICEGPU_AFFINE_SF>::pix(warps);
    *pix = SmemPlan<DICEGPU_AFFINE_SF>::pix_bytes(cap);
  }
}

static FrameKernelFn frame_fn(const dicegpu_ctx* c) {
  const bool dg = c->params.use_def_gradients != 0;
  return pick_frame_kernel(c->dp.shape, c->dp.interp, dg, c->use_masks);
}

static void fill_args(dicegpu_ctx* c, FrameArgs& a, int mode) {
  std::memset(&a, 0, sizeof(a));
  a.P = c->dp;
  a.ref = DevImage{c->W, c->H, c->d_ref, c->d_ref_gx, c->d_ref_gy, nullptr};
  a.def = DevImage{c->W, c->H, c->d_def, c->params.use_def_gradients ? c->d_def_gx : c->d_ref_gx,
                   c->params.use_def_gradients ? c->d_def_gy : c->d_ref_gy,
                   c->params.use_def_gradients ? c->d_def4 : nullptr};
  a.geo.half = c->use_lists ? -1 : c->params.subset_size / 2;
  a.geo.offsets = c->use_lists ? c->d_offsets : nullptr;
  a.geo.px = c->use_lists ? c->d_px : nullptr;
  a.geo.py = c->use_lists ? c->d_py : nullptr;
  a.geo.force_simplex = c->use_force ? c->d_force : nullptr;
  a.geo.mask_desc = c->use_masks ? c->d_mask_desc.p : nullptr;
  a.geo.mask_bits = c->d_mask_bits.p;
  a.geo.blocked_poly = c->d_bpoly.p;
  a.geo.blocked_vx = c->d_dvx.p;
  a.geo.blocked_vy = c->d_dvy.p;
  a.geo.pix_flag = c->has_evo ? c->d_pix_flag.p : nullptr;
  a.geo.pix_f = c->has_evo ? c->d_pix_f.p : nullptr;
  a.geo.evo_nact = c->has_evo ? c->d_evo_nact.p : nullptr;
  // turned on from the third frame of a sequence (frame_id_ > first_frame_id_
  // + frame_skip_, DICe_Schema.cpp:2357), in the tracking routine, whose
  // objectives persist across frames (DICe_Schema.cpp:1729-1748)
  a.evolve = c->has_evo && !c->evo_suspend && c->params.use_subset_evolution &&
             c->params.correlation_routine == DICEGPU_TRACKING_ROUTINE && c->frame_index >= 2;
  a.fields = c->d_fields;
  a.n = c->n;
  a.npix_cap = pix_cap(npix_max(c));
  a.pix_scratch = c->pix_in_global ? c->d_pix_scratch.p : nullptr;
  a.pix_stride = c->pix_stride;
  a.first_frame = c->frame_index == 0;
  a.mode = mode;
  a.plain_index = -1;
  a.work_counter = c->d_counter;
  a.queue_mode = c->queue_mode;
  a.chunk = c->chunk > 0 ? c->chunk : 4;
  a.status = c->d_status;
  a.passes_out = c->d_passes;
  a.unc = (c->params.compute_uncertainty && c->unc_n == c->n) ? c->d_unc : nullptr;
}

static int grid_for(dicegpu_ctx* c, FrameKernelFn fn, int* blocks, size_t* smem) {
  if (!fn) return DICEGPU_ERR_UNSUPPORTED;
  const int threads = c->warps_per_cta * 32;
  size_t fixed, pix;
  frame_smem_bytes(c, c->warps_per_cta, &fixed, &pix);
  // a subset's pixel arrays live in the CTA's shared memory, or, for subsets
  // too large for it, in a slice of a global scratch buffer per CTA
  c->pix_in_global = fixed + pix > (size_t)c->smem_optin;
  *smem = c->pix_in_global ? fixed : fixed + pix;
  c->pix_stride = pix;
  CK(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem));
  if (c->carveout >= 0)
    CK(cudaFuncSetAttribute((const void*)fn, cudaFuncAttributePreferredSharedMemoryCarveout, c->carveout));
  int per_sm = c->ctas_per_sm;
  if (per_sm <= 0) {
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, threads, *smem));
    if (per_sm < 1) per_sm = 1;
  }
  *blocks = std::min(per_sm * c->num_sms, kMaxQueues);
  if (c->pix_in_global) {
    int rc = c->d_pix_scratch.ensure((size_t)*blocks * pix);
    if (rc) return rc;
  }
  return DICEGPU_OK;
}

static int ready(dicegpu_ctx* c) {
  if (!c) return DICEGPU_ERR_ARG;
  if (!c->has_ref || !c->has_def || c->n < 1) return DICEGPU_ERR_STATE;
  if (!c->use_lists && c->params.subset_size < 1) return DICEGPU_ERR_ARG;
  return DICEGPU_OK;
}

// Per-frame state around the correlation kernels: at the first frame of a
// sequence the evolution state and the accumulated displacements restart;
// later frames of an incremental sequence zero the displacements first.
static int frame_begin(dicegpu_ctx* c) {
  const int n = c->n;
  const bool incr = c->params.use_incremental_formulation != 0;
  if (c->frame_index == 0) {
    if (c->has_evo) {
      CK(cudaMemcpyAsync(c->d_pix_flag.p, c->d_pix_flag0.p, c->evo_total, cudaMemcpyDeviceToDevice, c->stream));
      CK(cudaMemsetAsync(c->d_pix_f.p, 0, c->evo_total * sizeof(float), c->stream));
      CK(cudaMemcpyAsync(c->d_evo_nact.p, c->d_evo_nact0.p, (size_t)n * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                         c->stream));
    }
    if (incr) {
      int rc = c->d_acc.ensure(2 * (size_t)n);
      if (rc) return rc;
      CK(cudaMemsetAsync(c->d_acc.p, 0, 2 * (size_t)n * sizeof(double), c->stream));
    }
    return DICEGPU_OK;
  }
  if (incr) {
    if (!c->d_acc.p || c->d_acc.cap < 2 * (size_t)n) return DICEGPU_ERR_STATE;
    incr_begin_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(c->d_fields, n);
    CK(cudaGetLastError());
    c->launches += 1;
    if (c->has_evo && c->params.correlation_routine == DICEGPU_TRACKING_ROUTINE) {
      evo_rebase_kernel<<<(unsigned)((c->evo_total + 255) / 256), 256, 0, c->stream>>>(c->d_pix_flag.p,
                                                                                      c->evo_total);
      CK(cudaGetLastError());
      c->launches += 1;
    }
  }
  return DICEGPU_OK;
}

static int frame_end(dicegpu_ctx* c) {
  if (c->frame_index > 0 && c->params.use_incremental_formulation) {
    incr_end_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->d_fields, c->d_acc.p, c->n);
    CK(cudaGetLastError());
    c->launches += 1;
  }
  c->frame_index += 1;
  return DICEGPU_OK;
}

// Dependency waves of a frame (plan kind: bit 0 blocking subsets under the
// tracking routine, bit 1 neighbour initialization).  The reference runs the
// subsets in index order, so a subset depends on the blockers and the
// neighbour that precede it: level(i) = 1 + the largest level among them,
// and wave L holds the subsets of level L in index order.  Counting sort, O(n).
static int build_plan(dicegpu_ctx* c, int kind) {
  dicegpu_ctx::Plan& pl = c->plans[kind];
  if (pl.valid) return DICEGPU_OK;
  const int n = c->n;
  const bool blk = (kind & 1) && c->has_blocking && (int)c->h_blk_off.size() == n + 1;
  const bool nbr = (kind & 2) && (int)c->h_neigh.size() == n;
  std::vector<int32_t> level(n, 0);
  int nlev = 1;
  for (int i = 0; i < n; ++i) {
    int L = 0;
    if (blk)
      for (int k = c->h_blk_off[i]; k < c->h_blk_off[i + 1]; ++k) {
        const int j = c->h_blk_ids[k];
        if (j < i) L = std::max(L, level[j] + 1);
      }
    if (nbr) {
      const int j = c->h_neigh[i];
      if (j >= 0 && j < i) L = std::max(L, level[j] + 1);
    }
    level[i] = L;
    nlev = std::max(nlev, L + 1);
  }
  std::vector<int32_t> wave(n), wave_off(nlev + 1, 0), bwave_off(nlev + 1, 0), bwave;
  for (int i = 0; i < n; ++i) {
    ++wave_off[level[i] + 1];
    if (blk && (int)c->h_has_polys.size() == n && c->h_has_polys[i]) ++bwave_off[level[i] + 1];
  }
  for (int L = 0; L < nlev; ++L) {
    wave_off[L + 1] += wave_off[L];
    bwave_off[L + 1] += bwave_off[L];
  }
  bwave.resize(bwave_off[nlev]);
  {
    std::vector<int32_t> wf(wave_off.begin(), wave_off.end() - 1), bf(bwave_off.begin(), bwave_off.end() - 1);
    for (int i = 0; i < n; ++i) {
      wave[wf[level[i]]++] = i;
      if (blk && (int)c->h_has_polys.size() == n && c->h_has_polys[i]) bwave[bf[level[i]]++] = i;
    }
  }
  int rc;
  if ((rc = pl.d_wave.ensure(n)) || (rc = pl.d_bwave.ensure(std::max<size_t>(bwave.size(), 1)))) return rc;
  CK(cudaMemcpy(pl.d_wave.p, wave.data(), n * sizeof(int32_t), cudaMemcpyHostToDevice));
  if (!bwave.empty())
    CK(cudaMemcpy(pl.d_bwave.p, bwave.data(), bwave.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
  pl.wave_off.swap(wave_off);
  pl.bwave_off.swap(bwave_off);
  pl.valid = true;
  return DICEGPU_OK;
}

// The plan kind of the next frame (0: one launch over all subsets).
static int frame_plan_kind(const dicegpu_ctx* c) {
  int kind = 0;
  if (c->has_blocking && c->params.correlation_routine == DICEGPU_TRACKING_ROUTINE) kind |= 1;
  const int im = c->params.initialization_method;
  if ((int)c->h_neigh.size() == c->n &&
      (im == DICEGPU_USE_NEIGHBOR_VALUES || (im == DICEGPU_USE_NEIGHBOR_VALUES_FIRST_STEP_ONLY && c->frame_index == 0)))
    kind |= 2;
  return kind;
}

// A frame in dependency waves.  Blocked subsets get their blocked polygons
// rebuilt before their wave from their blockers' parameters (this frame's
// for lower indices, the frame-start snapshot's for higher ones); neighbour
// initialization reads the same way.  Runs of waves that hold a single
// subset without blocked polygons (a neighbour chain) go to one launch of
// a single warp, which takes them in order.  Everything is enqueued.
// A chain of single-subset waves runs alone on the GPU, one subset after the
// other: unless the caller chose the launch shape, its CTA takes the most
// warps the frame kernel allows (the passes and sweeps split over more warps;
// the sequential sums and the solve do not), when their shared memory fits.
static void chain_shape(dicegpu_ctx* c, FrameKernelFn fn, int* warps, size_t* smem) {
  const int w = DG_MAX_THREADS / 32;
  if (c->shape_set || w <= *warps) return;
  size_t fixed, pix;
  frame_smem_bytes(c, w, &fixed, &pix);
  const size_t s = c->pix_in_global ? fixed : fixed + pix;
  if (s > (size_t)c->smem_optin) return;
  if (s > *smem &&
      cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s) != cudaSuccess)
    return;
  *warps = w;
  *smem = s;
}

// A launch with few subsets per CTA (at most 6 per CTA of the default shape):
// unless the caller chose the launch shape, its CTAs take the kernel's most
// warps, so that each subset's passes and sweeps split further and the last
// subsets of the launch finish sooner.  Measured on a 2,500-subset conformal
// tracking frame: 3.05 ms per frame at four warps per CTA, 2.82 ms at eight;
// the 158,404-subset frame is faster at four.
static void wide_launch(dicegpu_ctx* c, FrameKernelFn fn, long n, int* warps, int* blocks, size_t* smem) {
  const int w = DG_MAX_THREADS / 32;
  if (c->shape_set || w <= *warps || n > 6L * *blocks) return;
  size_t fixed, pix;
  frame_smem_bytes(c, w, &fixed, &pix);
  const size_t s = c->pix_in_global ? fixed : fixed + pix;
  if (s > (size_t)c->smem_optin) return;
  if (s > *smem &&
      cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s) != cudaSuccess)
    return;
  if (c->wide_fn != (const void*)fn || c->wide_smem != s) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void*)fn, w * 32, s) != cudaSuccess)
      per_sm = 0;
    c->wide_fn = (const void*)fn;
    c->wide_smem = s;
    c->wide_per_sm = per_sm;
  }
  const int per_sm = c->wide_per_sm;
  if (per_sm < 1) return;
  *warps = w;
  *blocks = std::min(std::min(per_sm * c->num_sms, kMaxQueues), *blocks);
  *smem = s;
}

static int run_waves(dicegpu_ctx* c, int kind, FrameKernelFn fn, int blocks, size_t smem) {
  int rc;
  if ((kind & 1) && (rc = ensure_blocking_desc(c))) return rc;
  if ((rc = build_plan(c, kind))) return rc;
  const dicegpu_ctx::Plan& pl = c->plans[kind];
  const int n = c->n;
  if ((rc = c->d_snapshot.ensure((size_t)n * DICEGPU_FIELD_STRIDE))) return rc;
  CK(cudaMemcpyAsync(c->d_snapshot.p, c->d_fields, (size_t)n * DICEGPU_FIELD_STRIDE * sizeof(double),
                     cudaMemcpyDeviceToDevice, c->stream));
  BlockArgs ba;
  std::memset(&ba, 0, sizeof(ba));
  if (kind & 1) {
    ba.P = c->dp;
    ba.shapes = c->d_shapes.p;
    ba.shape_off = c->d_shape_off.p;
    ba.vx = c->d_svx.p;
    ba.vy = c->d_svy.p;
    ba.fields = c->d_fields;
    ba.snapshot = c->d_snapshot.p;
    ba.blk_off = c->d_blk_off.p;
    ba.blk_ids = c->d_blk_ids.p;
    ba.conformal = c->d_conformal.p;
    ba.dv_off = c->d_dv_off.p;
    ba.dp_off = c->d_dp_off.p;
    ba.dvx = c->d_dvx.p;
    ba.dvy = c->d_dvy.p;
    ba.polys = c->d_bpoly.p;
    ba.desc = c->d_mask_desc.p;
    ba.skin = (float)c->params.obstruction_skin_factor;
  }
  const int nlev = (int)pl.wave_off.size() - 1;
  for (int L = 0; L < nlev;) {
    const int nb = pl.bwave_off[L + 1] - pl.bwave_off[L];
    const int nw = pl.wave_off[L + 1] - pl.wave_off[L];
    FrameArgs a;
    fill_args(c, a, MODE_CORRELATE);
    if (kind & 2) {
      a.neigh = c->d_neigh.p;
      a.nsnap = c->d_snapshot.p;
    }
    if (nw == 1 && nb == 0) {
      // a chain: consecutive single-subset waves without blocked polygons,
      // taken in order by one CTA (all its warps on each subset)
      int L1 = L + 1;
      while (L1 < nlev && pl.wave_off[L1 + 1] - pl.wave_off[L1] == 1 && pl.bwave_off[L1 + 1] == pl.bwave_off[L1])
        ++L1;
      a.order = pl.d_wave.p + pl.wave_off[L];
      a.n_order = pl.wave_off[L1] - pl.wave_off[L];
      a.queue_mode = 0;
      int cw = c->warps_per_cta;
      size_t csmem = smem;
      chain_shape(c, fn, &cw, &csmem);
      CK(cudaMemsetAsync(c->d_counter, 0, sizeof(int), c->stream));
      fn<<<1, cw * 32, csmem, c->stream>>>(a);
      CK(cudaGetLastError());
      c->launches += 1;
      L = L1;
      continue;
    }
    if (nb > 0) {
      ba.list = pl.d_bwave.p + pl.bwave_off[L];
      ba.nlist = nb;
      const unsigned g = (unsigned)std::min((nb * 32 + 255) / 256, 8 * c->num_sms);   // a warp per subset
      if (c->dp.shape == DICEGPU_QUADRATIC_SF) blocked_kernel<DICEGPU_QUADRATIC_SF><<<g, 256, 0, c->stream>>>(ba);
      else blocked_kernel<DICEGPU_AFFINE_SF><<<g, 256, 0, c->stream>>>(ba);
      CK(cudaGetLastError());
      c->launches += 1;
    }
    if (nw > 0) {
      a.order = pl.d_wave.p + pl.wave_off[L];
      a.n_order = nw;
      int ww = c->warps_per_cta, wb = blocks;
      size_t ws = smem;
      wide_launch(c, fn, nw, &ww, &wb, &ws);
      CK(cudaMemsetAsync(c->d_counter, 0, (size_t)wb * sizeof(int), c->stream));
      fn<<<wb, ww * 32, ws, c->stream>>>(a);
      CK(cudaGetLastError());
      c->launches += 1;
    }
    ++L;
  }
  return DICEGPU_OK;
}

extern "C" int dicegpu_execute_correlation(dicegpu_ctx* c) {
  int rc = ready(c);
  if (rc) return rc;
  FrameKernelFn fn = frame_fn(c);
  int blocks;
  size_t smem;
  if ((rc = grid_for(c, fn, &blocks, &smem))) return rc;
  if ((rc = frame_begin(c))) return rc;
  const int kind = frame_plan_kind(c);
  if (kind) {
    if ((rc = run_waves(c, kind, fn, blocks, smem))) return rc;
    return frame_end(c);
  }
  FrameArgs a;
  fill_args(c, a, MODE_CORRELATE);
  int warps = c->warps_per_cta;
  wide_launch(c, fn, c->n, &warps, &blocks, &smem);
  CK(cudaMemsetAsync(c->d_counter, 0, (size_t)blocks * sizeof(int), c->stream));
  fn<<<blocks, warps * 32, smem, c->stream>>>(a);
  CK(cudaGetLastError());
  c->launches += 1;
  return frame_end(c);
}

extern "C" int dicegpu_execute_correlation_plain(dicegpu_ctx* c) {
  int rc = ready(c);
  if (rc) return rc;
  if (c->has_blocking && c->params.correlation_routine == DICEGPU_TRACKING_ROUTINE)
    return DICEGPU_ERR_UNSUPPORTED;
  FrameKernelFn fn = frame_fn(c);
  int blocks;
  size_t smem;
  if ((rc = grid_for(c, fn, &blocks, &smem))) return rc;
  if ((rc = frame_begin(c))) return rc;
  FrameArgs a;
  fill_args(c, a, MODE_CORRELATE);
  if (frame_plan_kind(c) & 2) {
    // launches in index order: a higher neighbour has not run yet
    a.neigh = c->d_neigh.p;
    a.nsnap = c->d_fields;
  }
  int warps = c->warps_per_cta;
  wide_launch(c, fn, 1, &warps, &blocks, &smem);
  for (int i = 0; i < c->n; ++i) {
    a.plain_index = i;
    fn<<<1, warps * 32, smem, c->stream>>>(a);
  }
  CK(cudaGetLastError());
  c->launches += c->n;
  return frame_end(c);
}

// ---------------------------------------------------------------------------
// frame sequences as CUDA graphs
// ---------------------------------------------------------------------------
extern "C" int dicegpu_capture_sequence(dicegpu_ctx* c, int n, const float* const* frames,
                                        const double* reset_fields) {
  if (!c || n < 1 || !frames) return DICEGPU_ERR_ARG;
  for (int k = 0; k < n; ++k)
    if (!frames[k]) return DICEGPU_ERR_ARG;
  if (!c->has_ref || c->n < 1) return DICEGPU_ERR_STATE;
  if (!c->cap_stream) CK(cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking));
  // everything a captured frame needs is allocated and uploaded first
  // (allocations and synchronous copies cannot be captured): blocking
  // descriptors, the wave plans of the first and the later frames, the
  // snapshot and the accumulated displacements
  {
    int rcb = DICEGPU_OK;
    if (c->has_blocking && c->params.correlation_routine == DICEGPU_TRACKING_ROUTINE) rcb = ensure_blocking_desc(c);
    const int saved = c->frame_index;
    for (int fi : {reset_fields ? 0 : saved, std::max(saved, 1)}) {
      c->frame_index = fi;
      const int kind = frame_plan_kind(c);
      if (!rcb && kind) rcb = build_plan(c, kind);
    }
    c->frame_index = saved;
    if (!rcb) rcb = c->d_snapshot.ensure((size_t)c->n * DICEGPU_FIELD_STRIDE);
    if (!rcb && c->params.use_incremental_formulation) rcb = c->d_acc.ensure(2 * (size_t)c->n);
    if (rcb) return rcb;
  }
  CK(cudaStreamSynchronize(c->stream));
  // an incremental sequence replays from the reference it was captured with
  const bool incr = c->params.use_incremental_formulation != 0;
  const size_t npx = (size_t)c->W * c->H;
  if (incr && reset_fields) {
    const int rcs = c->d_ref_saved.ensure(3 * npx);
    if (rcs) return rcs;
    CK(cudaMemcpy(c->d_ref_saved.p, c->d_ref, npx * sizeof(float), cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(c->d_ref_saved.p + npx, c->d_ref_gx, npx * sizeof(float), cudaMemcpyDeviceToDevice));
    CK(cudaMemcpy(c->d_ref_saved.p + 2 * npx, c->d_ref_gy, npx * sizeof(float), cudaMemcpyDeviceToDevice));
  }
  if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
  if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
  // record on a private stream; every call below only enqueues work
  cudaStream_t user_stream = c->stream;
  const int saved_frame = c->frame_index;
  const long long saved_launches = c->launches;
  const bool saved_has_def = c->has_def;
  c->stream = c->cap_stream;
  if (cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    c->stream = user_stream;
    return DICEGPU_ERR_CUDA;
  }
  int rc = DICEGPU_OK;
  if (reset_fields) {
    if (cudaMemcpyAsync(c->d_fields, reset_fields, (size_t)c->n * DICEGPU_FIELD_STRIDE * sizeof(double),
                        cudaMemcpyDeviceToDevice, c->cap_stream) != cudaSuccess)
      rc = DICEGPU_ERR_CUDA;
    c->frame_index = 0;
    if (incr && rc == DICEGPU_OK) {
      float* planes[3] = {c->d_ref, c->d_ref_gx, c->d_ref_gy};
      for (int q = 0; q < 3 && rc == DICEGPU_OK; ++q)
        if (cudaMemcpyAsync(planes[q], c->d_ref_saved.p + q * npx, npx * sizeof(float), cudaMemcpyDeviceToDevice,
                            c->cap_stream) != cudaSuccess)
          rc = DICEGPU_ERR_CUDA;
    }
  }
  for (int k = 0; k < n && rc == DICEGPU_OK; ++k) {
    if (incr && c->frame_index > 0) rc = dicegpu_set_ref_from_def(c);
    if (rc == DICEGPU_OK) rc = dicegpu_set_def_image(c, c->W, c->H, frames[k], 1);
    if (rc == DICEGPU_OK) rc = dicegpu_execute_correlation(c);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e = cudaStreamEndCapture(c->cap_stream, &g);
  c->stream = user_stream;
  c->frame_index = saved_frame;
  const long long per_replay = c->launches - saved_launches;
  c->launches = saved_launches;
  if (rc != DICEGPU_OK || e != cudaSuccess || !g) {
    if (g) cudaGraphDestroy(g);
    c->has_def = saved_has_def;
    return rc != DICEGPU_OK ? rc : DICEGPU_ERR_CUDA;
  }
  if (cudaGraphInstantiate(&c->graph_exec, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    c->graph_exec = nullptr;
    return DICEGPU_ERR_CUDA;
  }
  c->graph = g;
  c->graph_launches = per_replay;
  return DICEGPU_OK;
}

extern "C" int dicegpu_launch_sequence(dicegpu_ctx* c) {
  if (!c) return DICEGPU_ERR_ARG;
  if (!c->graph_exec) return DICEGPU_ERR_STATE;
  CK(cudaGraphLaunch(c->graph_exec, c->stream));
  c->launches += c->graph_launches;
  c->frame_index = 1;   // later frames continue the sequence
  return DICEGPU_OK;
}

// ---------------------------------------------------------------------------
// launch-shape autotuner
// ---------------------------------------------------------------------------
namespace {
struct TuneKey {
  int dev, shape, interp, defgrad, subset;
  bool operator<(const TuneKey& o) const {
    if (dev != o.dev) return dev < o.dev;
    if (shape != o.shape) return shape < o.shape;
    if (interp != o.interp) return interp < o.interp;
    if (defgrad != o.defgrad) return defgrad < o.defgrad;
    return subset < o.subset;
  }
};
struct TuneVal {
  int warps, ctas;
  float ms;
};
std::mutex g_tune_mu;
std::map<TuneKey, TuneVal> g_tune_cache;
}  // namespace

extern "C" int dicegpu_autotune(dicegpu_ctx* c, int* warps_per_cta, int* ctas_per_sm, float* best_ms) {
  int rc = ready(c);
  if (rc) return rc;
  const TuneKey key{c->device, c->dp.shape, c->dp.interp, c->params.use_def_gradients,
                    c->use_lists ? -1 : c->params.subset_size};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      c->warps_per_cta = it->second.warps;
      c->ctas_per_sm = it->second.ctas;
      c->shape_set = true;
      if (warps_per_cta) *warps_per_cta = it->second.warps;
      if (ctas_per_sm) *ctas_per_sm = it->second.ctas;
      if (best_ms) *best_ms = it->second.ms;
      return DICEGPU_OK;
    }
  }
  const size_t fb = (size_t)c->n * DICEGPU_FIELD_STRIDE * sizeof(double);
  double* saved = nullptr;
  if (cudaMalloc(&saved, fb) != cudaSuccess) return DICEGPU_ERR_NOMEM;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  rc = DICEGPU_OK;
  if (cudaMemcpyAsync(saved, c->d_fields, fb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess ||
      cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
    rc = DICEGPU_ERR_CUDA;
  const int frame0 = c->frame_index;
  c->evo_suspend = true;
  c->shape_set = true;   // each candidate runs with exactly its shape
  const int cand[][2] = {{4, 0}, {2, 0}, {8, 0}, {1, 0}, {4, 3}, {2, 6}};
  TuneVal best{c->warps_per_cta, c->ctas_per_sm, 1e30f};
  for (const auto& cd : cand) {
    if (rc) break;
    c->warps_per_cta = cd[0];
    c->ctas_per_sm = cd[1];
    float ms = 0.0f;
    for (int rep = 0; rep < 2 && !rc; ++rep) {   // first run warms the configuration up
      if (cudaMemcpyAsync(c->d_fields, saved, fb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess) {
        rc = DICEGPU_ERR_CUDA;
        break;
      }
      c->frame_index = frame0;
      cudaEventRecord(e0, c->stream);
      rc = dicegpu_execute_correlation(c);
      cudaEventRecord(e1, c->stream);
      if (!rc && cudaEventSynchronize(e1) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
      if (!rc) cudaEventElapsedTime(&ms, e0, e1);
    }
    if (!rc && ms < best.ms) best = TuneVal{cd[0], cd[1], ms};
  }
  // leave the fields and the sequence position as they were
  if (cudaMemcpyAsync(c->d_fields, saved, fb, cudaMemcpyDeviceToDevice, c->stream) != cudaSuccess && !rc)
    rc = DICEGPU_ERR_CUDA;
  cudaStreamSynchronize(c->stream);
  c->frame_index = frame0;
  c->evo_suspend = false;
  c->warps_per_cta = best.warps;
  c->ctas_per_sm = best.ctas;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(saved);
  if (rc) return rc;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache[key] = best;
  }
  if (warps_per_cta) *warps_per_cta = best.warps;
  if (ctas_per_sm) *ctas_per_sm = best.ctas;
  if (best_ms) *best_ms = best.ms;
  return DICEGPU_OK;
}

extern "C" int dicegpu_launch_count(dicegpu_ctx* c, int64_t* count) {
  if (!c || !count) return DICEGPU_ERR_ARG;
  *count = c->launches;
  return DICEGPU_OK;
}

extern "C" int dicegpu_set_launch_shape(dicegpu_ctx* c, int warps_per_cta, int ctas_per_sm) {
  if (!c || warps_per_cta < 0 || warps_per_cta > 8 || ctas_per_sm < 0) return DICEGPU_ERR_ARG;
  if (warps_per_cta > 0) c->warps_per_cta = warps_per_cta;
  if (ctas_per_sm >= 0) c->ctas_per_sm = ctas_per_sm;
  if (warps_per_cta > 0 || ctas_per_sm > 0) c->shape_set = true;
  return DICEGPU_OK;
}

extern "C" int dicegpu_get_launch_shape(dicegpu_ctx* c, int* warps_per_cta, int* ctas_per_sm) {
  if (!c || !warps_per_cta || !ctas_per_sm) return DICEGPU_ERR_ARG;
  *warps_per_cta = c->warps_per_cta;
  *ctas_per_sm = c->ctas_per_sm;
  return DICEGPU_OK;
}

extern "C" int dicegpu_device_status(dicegpu_ctx* c, int32_t* status) {
  if (!c || !status) return DICEGPU_ERR_ARG;
  CK(cudaMemcpyAsync(status, c->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return DICEGPU_OK;
}

extern "C" int dicegpu_gamma(dicegpu_ctx* c, const double* fields, double* gamma_out) {
  int rc = ready(c);
  if (rc) return rc;
  if (!fields || !gamma_out) return DICEGPU_ERR_ARG;
  double* d_f = nullptr;
  double* d_g = nullptr;
  const size_t fb = (size_t)c->n * DICEGPU_FIELD_STRIDE * sizeof(double);
  if (cudaMalloc(&d_f, fb) != cudaSuccess) return DICEGPU_ERR_NOMEM;
  if (cudaMalloc(&d_g, c->n * sizeof(double)) != cudaSuccess) { cudaFree(d_f); return DICEGPU_ERR_NOMEM; }
  rc = DICEGPU_OK;
  if (cudaMemcpyAsync(d_f, fields, fb, cudaMemcpyHostToDevice, c->stream) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
  FrameKernelFn fn = frame_fn(c);
  int blocks;
  size_t smem;
  if (!rc) rc = grid_for(c, fn, &blocks, &smem);
  if (!rc) {
    FrameArgs a;
    fill_args(c, a, MODE_GAMMA);
    a.fields = d_f;
    a.gamma_out = d_g;
    a.passes_out = nullptr;
    if (cudaMemsetAsync(c->d_counter, 0, (size_t)blocks * sizeof(int), c->stream) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
    fn<<<blocks, c->warps_per_cta * 32, smem, c->stream>>>(a);
    if (cudaGetLastError() != cudaSuccess) rc = DICEGPU_ERR_CUDA;
    c->launches += 1;
    if (!rc && cudaMemcpyAsync(gamma_out, d_g, c->n * sizeof(double), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      rc = DICEGPU_ERR_CUDA;
    if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
  }
  cudaStreamSynchronize(c->stream);
  cudaFree(d_f);
  cudaFree(d_g);
  return rc;
}

// One Objective entry point for every subset at the parameters of the
// caller's field rows (host memory).  MODE_GN / MODE_SIMPLEX write the
// updated shape-function fields back into `fields` plus iterations and
// Status_Flag per subset; MODE_SIGMA writes sigma and noise per subset.
static int run_objective_mode(dicegpu_ctx* c, int mode, double* fields, int32_t* iters,
                              int32_t* status, double* sigma, double* noise) {
  int rc = ready(c);
  if (rc) return rc;
  const size_t n = (size_t)c->n;
  const size_t fb = n * DICEGPU_FIELD_STRIDE * sizeof(double);
  const bool fit = mode == MODE_GN || mode == MODE_SIMPLEX;
  // one scratch block: fields | iterations | status | sigma | noise
  const size_t bytes = fb + 2 * n * sizeof(int32_t) + 2 * n * sizeof(double) + 64;
  unsigned char* buf = nullptr;
  if (cudaMalloc(&buf, bytes) != cudaSuccess) return DICEGPU_ERR_NOMEM;
  double* d_f = (double*)buf;
  int32_t* d_it = (int32_t*)(buf + fb);
  int32_t* d_st = d_it + n;
  double* d_sg = (double*)(((uintptr_t)(d_st + n) + 15) & ~(uintptr_t)15);
  double* d_no = d_sg + n;
  FrameKernelFn fn = frame_fn(c);
  int blocks;
  size_t smem;
  rc = grid_for(c, fn, &blocks, &smem);
  if (!rc && cudaMemcpyAsync(d_f, fields, fb, cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
    rc = DICEGPU_ERR_CUDA;
  if (!rc) {
    FrameArgs a;
    fill_args(c, a, mode);
    a.fields = d_f;
    a.passes_out = nullptr;
    a.iter_out = d_it;
    a.status_out = d_st;
    a.gamma_out = d_sg;
    a.noise_out = d_no;
    if (cudaMemsetAsync(c->d_counter, 0, (size_t)blocks * sizeof(int), c->stream) != cudaSuccess)
      rc = DICEGPU_ERR_CUDA;
    fn<<<blocks, c->warps_per_cta * 32, smem, c->stream>>>(a);
    if (cudaGetLastError() != cudaSuccess) rc = DICEGPU_ERR_CUDA;
    c->launches += 1;
  }
  auto d2h = [&](void* dst, const void* src, size_t b) {
    if (!rc && dst && cudaMemcpyAsync(dst, src, b, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      rc = DICEGPU_ERR_CUDA;
  };
  if (fit) {
    d2h(fields, d_f, fb);
    d2h(iters, d_it, n * sizeof(int32_t));
    d2h(status, d_st, n * sizeof(int32_t));
  } else {
    d2h(sigma, d_sg, n * sizeof(double));
    d2h(noise, d_no, n * sizeof(double));
  }
  if (cudaStreamSynchronize(c->stream) != cudaSuccess && !rc) rc = DICEGPU_ERR_CUDA;
  cudaFree(buf);
  return rc;
}

extern "C" int dicegpu_compute_update_fast(dicegpu_ctx* c, double* fields, int32_t* num_iterations,
                                           int32_t* status) {
  if (!c || !fields || !num_iterations || !status) return DICEGPU_ERR_ARG;
  return run_objective_mode(c, MODE_GN, fields, num_iterations, status, nullptr, nullptr);
}

extern "C" int dicegpu_compute_update_robust(dicegpu_ctx* c, double* fields, int32_t* num_iterations,
                                             int32_t* status) {
  if (!c || !fields || !num_iterations || !status) return DICEGPU_ERR_ARG;
  return run_objective_mode(c, MODE_SIMPLEX, fields, num_iterations, status, nullptr, nullptr);
}

extern "C" int dicegpu_sigma(dicegpu_ctx* c, const double* fields, double* sigma_out, double* noise_out) {
  if (!c || !fields || !sigma_out) return DICEGPU_ERR_ARG;
  return run_objective_mode(c, MODE_SIGMA, const_cast<double*>(fields), nullptr, nullptr, sigma_out,
                            noise_out);
}

extern "C" int dicegpu_adjoint(dicegpu_ctx* c, const double* d_fields, const double* d_seed,
                               int objective, int grad_source, double* d_value, double* d_dparams,
                               float* d_ddef) {
  int rc = ready(c);
  if (rc) return rc;
  if (!d_fields || objective < 0 || objective > 1 || grad_source < 0 || grad_source > 1)
    return DICEGPU_ERR_ARG;
  if (c->params.interpolation != DICEGPU_KEYS_FOURTH) return DICEGPU_ERR_UNSUPPORTED;
  if (grad_source == 1 && !c->params.use_def_gradients) return DICEGPU_ERR_STATE;
  AdjointArgs a;
  std::memset(&a, 0, sizeof(a));
  a.P = c->dp;
  a.ref = DevImage{c->W, c->H, c->d_ref, c->d_ref_gx, c->d_ref_gy, nullptr};
  a.def = DevImage{c->W, c->H, c->d_def, c->d_def_gx, c->d_def_gy, nullptr};
  a.geo.half = c->use_lists ? -1 : c->params.subset_size / 2;
  a.geo.offsets = c->use_lists ? c->d_offsets : nullptr;
  a.geo.px = c->use_lists ? c->d_px : nullptr;
  a.geo.py = c->use_lists ? c->d_py : nullptr;
  a.fields = d_fields;
  a.seed = d_seed;
  a.n = c->n;
  a.objective = objective;
  a.grad_source = grad_source;
  a.value_out = d_value;
  a.dparams_out = d_dparams;
  a.ddef = d_ddef;
  const void* fn = c->dp.shape == DICEGPU_QUADRATIC_SF ? (const void*)adjoint_kernel<DICEGPU_QUADRATIC_SF>
                                                      : (const void*)adjoint_kernel<DICEGPU_AFFINE_SF>;
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 256, 0));
  const int need = (c->n + 7) / 8;
  const int blocks = std::max(1, std::min(std::max(per_sm, 1) * c->num_sms, need));
  if (c->dp.shape == DICEGPU_QUADRATIC_SF)
    adjoint_kernel<DICEGPU_QUADRATIC_SF><<<blocks, 256, 0, c->stream>>>(a);
  else
    adjoint_kernel<DICEGPU_AFFINE_SF><<<blocks, 256, 0, c->stream>>>(a);
  CK(cudaGetLastError());
  c->launches += 1;
  return DICEGPU_OK;
}

extern "C" int dicegpu_interpolate(dicegpu_ctx* c, int method, int n, const float* xy,
                                   float* intensity, float* grad_x, float* grad_y, int on_device) {
  if (!c || !xy || !intensity || n < 0) return DICEGPU_ERR_ARG;
  if (!c->has_def) return DICEGPU_ERR_STATE;
  if (method < DICEGPU_BILINEAR || method > DICEGPU_KEYS_FOURTH) return DICEGPU_ERR_ARG;
  if (n == 0) return DICEGPU_OK;
  const bool grad = grad_x && grad_y && c->params.use_def_gradients;
  const float *dxy = xy;
  float *di = intensity, *dgx = grad_x, *dgy = grad_y;
  float* buf = nullptr;
  if (!on_device) {
    if (cudaMalloc(&buf, (size_t)n * 5 * sizeof(float)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
    dxy = buf;
    di = buf + 2 * (size_t)n;
    dgx = buf + 3 * (size_t)n;
    dgy = buf + 4 * (size_t)n;
    if (cudaMemcpyAsync((void*)dxy, xy, 2 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
      cudaFree(buf);
      return DICEGPU_ERR_CUDA;
    }
  }
  interp_kernel<<<(n + 255) / 256, 256, 0, c->stream>>>(
      method, c->W, c->H, c->d_def, grad ? c->d_def_gx : nullptr, grad ? c->d_def_gy : nullptr, n,
      dxy, di, grad ? dgx : nullptr, grad ? dgy : nullptr);
  c->launches += 1;
  int rc = cudaGetLastError() == cudaSuccess ? DICEGPU_OK : DICEGPU_ERR_CUDA;
  if (!on_device) {
    if (!rc && cudaMemcpyAsync(intensity, di, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
    if (!rc && grad) {
      if (cudaMemcpyAsync(grad_x, dgx, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
      if (cudaMemcpyAsync(grad_y, dgy, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess) rc = DICEGPU_ERR_CUDA;
    }
    cudaStreamSynchronize(c->stream);
    cudaFree(buf);
  }
  return rc;
}

extern "C" int dicegpu_image_gradients(int w, int h, const float* d_img, float* d_gx, float* d_gy,
                                       int method, void* stream) {
  if (!d_img || !d_gx || !d_gy || w < 3 || h < 3) return DICEGPU_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  float* tmp = nullptr;
  if (method == DICEGPU_CONVOLUTION_5_POINT) {
    if (cudaMalloc(&tmp, 2 * (size_t)w * h * sizeof(float)) != cudaSuccess) return DICEGPU_ERR_NOMEM;
  }
  int rc = launch_gradients(w, h, d_img, d_gx, d_gy, method, tmp, st, nullptr);
  if (tmp) {
    cudaStreamSynchronize(st);
    cudaFree(tmp);
  }
  return rc;
}

extern "C" int dicegpu_gauss_filter(int w, int h, const float* d_in, float* d_out, int mask_size,
                                    void* stream) {
  if (!d_in || !d_out || d_in == d_out || w < 1 || h < 1) return DICEGPU_ERR_ARG;
  return launch_gauss_filter(w, h, mask_size, d_in, d_out, (cudaStream_t)stream, nullptr);
}

// ---------------------------------------------------------------------------
// Gradients without any device allocation.
//
// For callers that cannot allocate device memory themselves: hosts that give
// the library a fixed device-memory budget owned by their own pool, or
// per-frame loops that cannot afford cudaMalloc / cudaFree (cudaFree waits
// for the whole device).  The two intermediate finite-difference planes that
// dicegpu_image_gradients allocates for the 5-point smoothing live instead in
// the file-scope array below, which every GPU that loads this library holds
// until the process exits (8 MiB).
// ---------------------------------------------------------------------------
static __device__ __align__(256) float g_noalloc_scratch[2 * DICEGPU_NOALLOC_MAX_PIXELS];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
float* g_noalloc_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the host-side symbol is only a stand-in for it).
int noalloc_scratch(float** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DICEGPU_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return DICEGPU_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return DICEGPU_ERR_CUDA;
    g_noalloc_ptr[dev] = static_cast<float*>(p);
  }
  *out = g_noalloc_ptr[dev];
  return DICEGPU_OK;
}
}  // namespace

extern "C" int dicegpu_image_gradients_noalloc(int w, int h, const float* d_img, float* d_gx,
                                               float* d_gy, int method, void* stream) {
  if (!d_img || !d_gx || !d_gy || w < 3 || h < 3) return DICEGPU_ERR_ARG;
  if (method != DICEGPU_FINITE_DIFFERENCE && method != DICEGPU_CONVOLUTION_5_POINT)
    return DICEGPU_ERR_ARG;
  float* tmp = nullptr;
  if (method == DICEGPU_CONVOLUTION_5_POINT) {
    // only the smoothing step needs the intermediate planes
    if ((long long)w * h > DICEGPU_NOALLOC_MAX_PIXELS) return DICEGPU_ERR_ARG;
    const int rc = noalloc_scratch(&tmp);
    if (rc) return rc;
  }
  // the finite-difference kernel writes every scratch element the smoothing
  // kernel reads, so nothing needs clearing between calls
  return launch_gradients(w, h, d_img, d_gx, d_gy, method, tmp, (cudaStream_t)stream, nullptr);
}

// dice_correlate's stride-9 interface (DICe_api.cpp:51-151).  As the
// reference keeps a static Schema, one context lives across calls: the first
// call creates it from the parameters (tracking_default_params when NULL,
// DICe_api.cpp:84-93), the subset size and coordinates, and the reference
// image; every call takes a new deformed image and the nine stride-9 columns
// of every subset, the other field columns carrying over from the previous
// call as the Schema's fields do; the parameters are read again only when
// update_params is set (DICe_api.cpp:114-115).  The frame count carries over
// too, so only the first call is the sequence's first frame.
namespace {
std::mutex g_api_mu;
dicegpu_ctx* g_api_ctx = nullptr;
int g_api_device = -1;
int g_api_subset = 0;
std::vector<double> g_api_rows;   // the context's field rows after the last call

int api_params(const dicegpu_params* in, int subset_size, dicegpu_params* p) {
  if (in) {
    *p = *in;
  } else {
    const int rc = dicegpu_tracking_default_params(p);
    if (rc) return rc;
  }
  // the api routines take the affine shape function only (DICe_api.cpp:116)
  if (p->shape_function != DICEGPU_AFFINE_SF) return DICEGPU_ERR_UNSUPPORTED;
  p->subset_size = subset_size;
  p->use_def_gradients = 1;   // arrays: Schema::set_def_image(w,h,array), DICe_Schema.cpp:339
  return DICEGPU_OK;
}

void api_release() {
  if (!g_api_ctx) return;
  int cur = -1;
  const bool restore = cudaGetDevice(&cur) == cudaSuccess && cur != g_api_device;
  if (restore) cudaSetDevice(g_api_device);
  dicegpu_destroy(g_api_ctx);
  if (restore) cudaSetDevice(cur);
  g_api_ctx = nullptr;
  g_api_device = -1;
  g_api_subset = 0;
  g_api_rows.clear();
}
}  // namespace

extern "C" int dicegpu_correlate(float* points, int n_points, int subset_size, const float* ref_img,
                                 int ref_w, int ref_h, const float* def_img, int def_w, int def_h,
                                 const dicegpu_params* params, int update_params) {
  if (ref_w != def_w || ref_h != def_h) return -1;
  if (subset_size < 1) return -1;
  if (n_points < 1) return -1;
  if (!points || !ref_img || !def_img) return -1;
  std::lock_guard<std::mutex> lock(g_api_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return DICEGPU_ERR_CUDA;
  int rc = DICEGPU_OK;
  const bool first = g_api_ctx == nullptr;
  if (first) {
    dicegpu_params p;
    rc = api_params(params, subset_size, &p);
    if (rc) return rc;
    rc = dicegpu_create(&p, &g_api_ctx);
    if (rc) return rc;
    g_api_device = dev;
    g_api_subset = subset_size;
    g_api_rows.assign((size_t)n_points * DICEGPU_FIELD_STRIDE, 0.0);
  } else {
    // the subsets are the first call's; a context made on another device
    // cannot be used from this one
    if ((size_t)n_points * DICEGPU_FIELD_STRIDE != g_api_rows.size()) return DICEGPU_ERR_ARG;
    if (dev != g_api_device) return DICEGPU_ERR_STATE;
    if (update_params) {
      dicegpu_params p;
      rc = api_params(params, g_api_subset, &p);
      if (!rc) rc = dicegpu_set_params(g_api_ctx, &p);
      if (rc) return rc;
    }
  }
  for (int i = 0; i < n_points; ++i) {
    double* r = &g_api_rows[(size_t)i * DICEGPU_FIELD_STRIDE];
    const float* q = points + (size_t)i * DICEGPU_API_STRIDE;
    r[DICEGPU_F_COORD_X] = q[0];
    r[DICEGPU_F_COORD_Y] = q[1];
    r[DICEGPU_F_DISP_X] = q[2];
    r[DICEGPU_F_DISP_Y] = q[3];
    r[DICEGPU_F_ROT_Z] = q[4];
    r[DICEGPU_F_SIGMA] = q[5];
    r[DICEGPU_F_GAMMA] = q[6];
    r[DICEGPU_F_BETA] = q[7];
    r[DICEGPU_F_STATUS] = q[8];
  }
  dicegpu_ctx* c = g_api_ctx;
  if (first) {
    rc = dicegpu_set_ref_image(c, ref_w, ref_h, ref_img, 0);
    if (!rc) rc = dicegpu_set_subsets(c, n_points, g_api_rows.data());
  } else if (cudaMemcpyAsync(c->d_fields, g_api_rows.data(), g_api_rows.size() * sizeof(double),
                             cudaMemcpyHostToDevice, c->stream) != cudaSuccess) {
    rc = DICEGPU_ERR_CUDA;   // (dicegpu_load_fields would restart the sequence)
  }
  if (!rc) rc = dicegpu_set_def_image(c, def_w, def_h, def_img, 0);
  if (!rc) rc = dicegpu_execute_correlation(c);
  if (!rc) rc = dicegpu_get_fields(c, g_api_rows.data());
  if (rc) {
    // a failed call leaves no half-made state behind
    api_release();
    return rc;
  }
  for (int i = 0; i < n_points; ++i) {
    const double* r = &g_api_rows[(size_t)i * DICEGPU_FIELD_STRIDE];
    float* q = points + (size_t)i * DICEGPU_API_STRIDE;
    q[2] = (float)r[DICEGPU_F_DISP_X];
    q[3] = (float)r[DICEGPU_F_DISP_Y];
    q[4] = (float)r[DICEGPU_F_ROT_Z];
    q[5] = (float)r[DICEGPU_F_SIGMA];
    q[6] = (float)r[DICEGPU_F_GAMMA];
    q[7] = (float)r[DICEGPU_F_BETA];
    q[8] = (float)r[DICEGPU_F_STATUS];
  }
  return DICEGPU_OK;
}

extern "C" int dicegpu_correlate_reset(void) {
  std::lock_guard<std::mutex> lock(g_api_mu);
  api_release();
  return DICEGPU_OK;
}

#ifdef DG_PROFILE
// profiling builds only: read and clear the section timers of every frame
// kernel unit (cycles summed over the units)
extern "C" int dicegpu_prof_read(unsigned long long* out16) {
  unsigned long long acc[16] = {};
  int bad = 0;
  bad |= DG_FRAME_PROF_NAME(0, 0, 0)(acc) | DG_FRAME_PROF_NAME(0, 1, 0)(acc) | DG_FRAME_PROF_NAME(0, 2, 0)(acc);
  bad |= DG_FRAME_PROF_NAME(1, 0, 0)(acc) | DG_FRAME_PROF_NAME(1, 1, 0)(acc) | DG_FRAME_PROF_NAME(1, 2, 0)(acc);
  bad |= DG_FRAME_PROF_NAME(0, 0, 1)(acc) | DG_FRAME_PROF_NAME(0, 1, 1)(acc) | DG_FRAME_PROF_NAME(0, 2, 1)(acc);
  bad |= DG_FRAME_PROF_NAME(1, 0, 1)(acc) | DG_FRAME_PROF_NAME(1, 1, 1)(acc) | DG_FRAME_PROF_NAME(1, 2, 1)(acc);
  std::memcpy(out16, acc, sizeof(acc));
  return bad ? DICEGPU_ERR_CUDA : DICEGPU_OK;
}
#endif
