// dg_frame.cuh -- the persistent frame kernel and its instantiation picker.
//
// frame_kernel<shape, interp, defgrad, mask> runs Schema::execute_correlation
// (or one Objective entry point, by mode) for every subset of a launch: one
// CTA per subset from interleaved per-CTA work queues.  The instantiations
// live in frame_inst.cu (one unit per shape function, interpolation and
// mask); the unmasked kernels are exactly what they are without masks.
#pragma once

#include "dg_engine.cuh"

// launch bounds of the frame kernel: at most DG_MAX_THREADS threads per CTA
// (warps per subset <= DG_MAX_THREADS / 32) and DG_MIN_BLOCKS resident CTAs
// of that size per SM, which bounds its registers
#ifndef DG_MAX_THREADS
#define DG_MAX_THREADS 256
#endif
#ifndef DG_MIN_BLOCKS
#define DG_MIN_BLOCKS 2
#endif

namespace dg {

// ---------------------------------------------------------------------------
// the persistent frame kernel: one CTA (up to 8 warps) per subset
// ---------------------------------------------------------------------------
template <int SHAPE, int INTERP, bool DEFGRAD, bool MASK>
__global__ void __launch_bounds__(DG_MAX_THREADS, DG_MIN_BLOCKS) frame_kernel(const __grid_constant__ FrameArgs a) {
  Engine<SHAPE, INTERP, DEFGRAD, MASK> e(a);
  Ctl& c = ctl();
  if (a.plain_index >= 0) {
    if (blockIdx.x == 0) e.run(a.plain_index);
    return;
  }
  // the launch's subsets: all n, or the n_order listed in order
  const int count = a.order ? a.n_order : a.n;
  if (a.queue_mode == 0) {
    // one global queue head
    for (;;) {
      if (threadIdx.x == 0) c.work = atomicAdd(a.work_counter, 1);
      __syncthreads();
      const int t = c.work;
      __syncthreads();
      if (t >= count) break;
      e.run(a.order ? a.order[t] : t);
    }
    return;
  }
  // Interleaved per-CTA queues: the subsets are cut into chunks of C
  // consecutive ones and CTA r owns chunks r, r + G, r + 2G, ...  All CTAs
  // advance through the image together (a narrow band resident in L2).  A
  // CTA whose chunks are exhausted takes from the following CTAs' sequences.
  // Every index is taken exactly once (atomicAdd); a CTA leaves after finding
  // all G sequences exhausted, so no CTA ever waits on another.
  const int G = gridDim.x;
  const int C = a.chunk;
  int q = blockIdx.x;
  for (int visited = 0; visited < G;) {
    if (threadIdx.x == 0) c.work = atomicAdd(a.work_counter + q, 1);
    __syncthreads();
    const int t = c.work;
    __syncthreads();
    const long long chunk = (long long)q + (long long)(t / C) * G;
    const long long lidx = chunk * C + (t % C);
    const int pos = lidx < count ? (int)lidx : count;
    if (pos < count) {
      DG_PT(t_run);
      e.run(a.order ? a.order[pos] : pos);
      DG_PACC(0, t_run);
      continue;
    }
    ++visited;
    q = (q + 1 == G) ? 0 : q + 1;
  }
}

typedef void (*FrameKernelFn)(FrameArgs);

// The frame kernels are instantiated in frame_inst.cu, compiled once per
// (shape function, interpolation, mask) so that the units build in
// parallel: frame_fn_s<shape>_i<interp>_m<mask>(defgrad) returns the kernel
// with or without deformed-image gradients.  MASK selects the instantiation
// whose passes test obstruction bitmaps and blocked polygons (only contexts
// with masks launch it).
#define DG_FRAME_FN_NAME(S, I, M) frame_fn_s##S##_i##I##_m##M
#define DG_DECLARE_FRAME_FN(S, I, M) FrameKernelFn DG_FRAME_FN_NAME(S, I, M)(bool defgrad);
DG_DECLARE_FRAME_FN(0, 0, 0) DG_DECLARE_FRAME_FN(0, 1, 0) DG_DECLARE_FRAME_FN(0, 2, 0)
DG_DECLARE_FRAME_FN(1, 0, 0) DG_DECLARE_FRAME_FN(1, 1, 0) DG_DECLARE_FRAME_FN(1, 2, 0)
DG_DECLARE_FRAME_FN(0, 0, 1) DG_DECLARE_FRAME_FN(0, 1, 1) DG_DECLARE_FRAME_FN(0, 2, 1)
DG_DECLARE_FRAME_FN(1, 0, 1) DG_DECLARE_FRAME_FN(1, 1, 1) DG_DECLARE_FRAME_FN(1, 2, 1)

#ifdef DG_PROFILE
// profiling builds: each unit adds its section timers into acc16 and clears them
#define DG_FRAME_PROF_NAME(S, I, M) frame_prof_s##S##_i##I##_m##M
#define DG_DECLARE_FRAME_PROF(S, I, M) int DG_FRAME_PROF_NAME(S, I, M)(unsigned long long* acc16);
DG_DECLARE_FRAME_PROF(0, 0, 0) DG_DECLARE_FRAME_PROF(0, 1, 0) DG_DECLARE_FRAME_PROF(0, 2, 0)
DG_DECLARE_FRAME_PROF(1, 0, 0) DG_DECLARE_FRAME_PROF(1, 1, 0) DG_DECLARE_FRAME_PROF(1, 2, 0)
DG_DECLARE_FRAME_PROF(0, 0, 1) DG_DECLARE_FRAME_PROF(0, 1, 1) DG_DECLARE_FRAME_PROF(0, 2, 1)
DG_DECLARE_FRAME_PROF(1, 0, 1) DG_DECLARE_FRAME_PROF(1, 1, 1) DG_DECLARE_FRAME_PROF(1, 2, 1)
#endif

// The frame kernel of a configuration (nullptr for one this build leaves
// out: a unit compiled with DG_ONLY_BENCH_KERNEL returns only the affine /
// Keys-4 / deformed-gradient kernel).
inline FrameKernelFn pick_frame_kernel(int shape, int interp, bool defgrad, bool mask) {
  typedef FrameKernelFn (*Pick)(bool);
  static const Pick table[2][3][2] = {
      {{DG_FRAME_FN_NAME(0, 0, 0), DG_FRAME_FN_NAME(0, 0, 1)},
       {DG_FRAME_FN_NAME(0, 1, 0), DG_FRAME_FN_NAME(0, 1, 1)},
       {DG_FRAME_FN_NAME(0, 2, 0), DG_FRAME_FN_NAME(0, 2, 1)}},
      {{DG_FRAME_FN_NAME(1, 0, 0), DG_FRAME_FN_NAME(1, 0, 1)},
       {DG_FRAME_FN_NAME(1, 1, 0), DG_FRAME_FN_NAME(1, 1, 1)},
       {DG_FRAME_FN_NAME(1, 2, 0), DG_FRAME_FN_NAME(1, 2, 1)}}};
  if (shape < 0 || shape > 1 || interp < 0 || interp > 2) return nullptr;
  return table[shape][interp][mask ? 1 : 0](defgrad);
}

}  // namespace dg
