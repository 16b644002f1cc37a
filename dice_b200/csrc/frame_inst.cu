// frame_inst.cu -- the frame kernels of one (shape function, interpolation,
// mask) combination, with and without deformed-image gradients.  The
// Makefile compiles this unit once per combination (DG_INST_SHAPE,
// DG_INST_INTERP, DG_INST_MASK), so the twelve units build in parallel.
#include "dg_frame.cuh"

#if !defined(DG_INST_SHAPE) || !defined(DG_INST_INTERP) || !defined(DG_INST_MASK)
#error "frame_inst.cu is compiled with DG_INST_SHAPE, DG_INST_INTERP and DG_INST_MASK"
#endif

namespace dg {

#define DG_CAT_FN(S, I, M) DG_FRAME_FN_NAME(S, I, M)
FrameKernelFn DG_CAT_FN(DG_INST_SHAPE, DG_INST_INTERP, DG_INST_MASK)(bool defgrad) {
#ifdef DG_ONLY_BENCH_KERNEL
  // reduced build (fast compiles while tuning): only the affine / Keys-4 /
  // deformed-gradient kernels
#if DG_INST_SHAPE == 0 && DG_INST_INTERP == 2
  return defgrad ? frame_kernel<DICEGPU_AFFINE_SF, DICEGPU_KEYS_FOURTH, true, DG_INST_MASK != 0> : nullptr;
#else
  (void)defgrad;
  return nullptr;
#endif
#else
  return defgrad ? frame_kernel<DG_INST_SHAPE, DG_INST_INTERP, true, DG_INST_MASK != 0>
                 : frame_kernel<DG_INST_SHAPE, DG_INST_INTERP, false, DG_INST_MASK != 0>;
#endif
}

#ifdef DG_PROFILE
#define DG_CAT_PROF(S, I, M) DG_FRAME_PROF_NAME(S, I, M)
int DG_CAT_PROF(DG_INST_SHAPE, DG_INST_INTERP, DG_INST_MASK)(unsigned long long* acc16) {
  unsigned long long v[16];
  if (cudaMemcpyFromSymbol(v, g_prof, sizeof(v)) != cudaSuccess) return 1;
  for (int i = 0; i < 16; ++i) acc16[i] += v[i];
  const unsigned long long z[16] = {};
  return cudaMemcpyToSymbol(g_prof, z, sizeof(z)) != cudaSuccess ? 1 : 0;
}
#endif

}  // namespace dg
