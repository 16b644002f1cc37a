// dg_frame.cuh -- the persistent frame kernel and its instantiation picker.
//
// frame_kernel<shape, interp, defgrad, mask> runs Schema::execute_correlation
// (or one Objective entry point, by mode) for every subset of a launch: one
// CTA per subset from interleaved per-CTA work queues.  The unmasked
// instantiations are compiled with the rest of the library (dicegpu.cu), the
// masked ones in frame_masked.cu, so that both compile in parallel and the
// unmasked kernels are exactly what they are without masks.
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

// The frame kernel of a configuration; MASK selects the instantiation whose
// passes test obstruction bitmaps and blocked polygons (only subsets with masks pay
// for it, and only contexts with masks launch it).
template <int SHAPE, bool MASK>
static FrameKernelFn pick_kernel(int interp, bool defgrad) {
#ifdef DG_ONLY_BENCH_KERNEL
  // reduced build (fast compiles while tuning): only the affine / Keys-4 /
  // deformed-gradient kernel; other configurations report UNSUPPORTED
  if (SHAPE == DICEGPU_AFFINE_SF && interp == DICEGPU_KEYS_FOURTH && defgrad)
    return frame_kernel<DICEGPU_AFFINE_SF, DICEGPU_KEYS_FOURTH, true, MASK>;
  return nullptr;
#else
  if (defgrad) {
    if (interp == DICEGPU_KEYS_FOURTH) return frame_kernel<SHAPE, DICEGPU_KEYS_FOURTH, true, MASK>;
    if (interp == DICEGPU_BICUBIC) return frame_kernel<SHAPE, DICEGPU_BICUBIC, true, MASK>;
    return frame_kernel<SHAPE, DICEGPU_BILINEAR, true, MASK>;
  }
  if (interp == DICEGPU_KEYS_FOURTH) return frame_kernel<SHAPE, DICEGPU_KEYS_FOURTH, false, MASK>;
  if (interp == DICEGPU_BICUBIC) return frame_kernel<SHAPE, DICEGPU_BICUBIC, false, MASK>;
  return frame_kernel<SHAPE, DICEGPU_BILINEAR, false, MASK>;
#endif
}

// the masked instantiations live in their own translation unit (frame_masked.cu)
FrameKernelFn pick_masked_kernel(int shape, int interp, bool defgrad);

}  // namespace dg
