// frame_masked.cu -- the frame kernels whose passes test obstruction and
// blocked bitmaps (contexts with obstructed shapes or blocking subsets).
#include "dg_frame.cuh"

namespace dg {

FrameKernelFn pick_masked_kernel(int shape, int interp, bool defgrad) {
  return shape == DICEGPU_QUADRATIC_SF ? pick_kernel<DICEGPU_QUADRATIC_SF, true>(interp, defgrad)
                                       : pick_kernel<DICEGPU_AFFINE_SF, true>(interp, defgrad);
}

}  // namespace dg
