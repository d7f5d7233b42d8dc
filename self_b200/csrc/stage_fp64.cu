// FP64 instantiation of the fused stage kernels.  Built with -fmad=false: no
// multiply-add contraction, and divisions and square roots are IEEE correctly
// rounded, so each value is formed with the same roundings as the reference's
// FP64 CPU path evaluated in the same order.
#include "stage_dispatch.cuh"

namespace selfgpu {
cudaError_t launch_stage_fp64(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                              int* usedTma) {
  return launch_stage_impl<double>(model, P, a, L, st, usedTma);
}
}  // namespace selfgpu
