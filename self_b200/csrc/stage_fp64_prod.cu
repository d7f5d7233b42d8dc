// Production FP64 instantiation of the fused stage kernels.  Built with
// multiply-add contraction; the surface lift multiplies by the reciprocal
// quadrature weights, the divergence by 1/J (held in the packed geometry
// record) and the point-wise state by one reciprocal of the density.  Every
// value stays FP64; results differ from the reference-rounding build
// (stage_fp64.cu) at the FP64 round-off level.
#define SELFGPU_FP64_PRODUCTION 1
#include "stage_dispatch.cuh"

namespace selfgpu {
cudaError_t launch_stage_fp64(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                              int* usedTma) {
  return launch_stage_impl<double>(model, P, a, L, st, usedTma);
}
cudaError_t launch_steps_fp64(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st) {
  return launch_steps_impl<double>(model, P, a, sa, numSMs, st);
}
cudaError_t launch_stages_tma_fp64(int model, int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                  cudaStream_t st) {
  return launch_stages_tma_impl<double>(model, P, a, L, ms, st);
}
}  // namespace selfgpu
