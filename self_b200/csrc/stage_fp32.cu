// FP32-bulk instantiation of the fused stage kernels: fluxes, traces and the
// divergence in float (with multiply-add contraction); metric terms, sources'
// fields and the RK accumulation of the solution stay in double.
#include "av_closure.cuh"
#include "stage_dispatch.cuh"

namespace selfgpu {
cudaError_t launch_stage_fp32(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                              int* usedTma) {
  return launch_stage_impl<float>(model, P, a, L, st, usedTma);
}
cudaError_t launch_av_prep_fp32(int P, const AvArgs& a, cudaStream_t st, int numSMs, bool formNu) {
  return launch_av_prep_impl<float>(P, a, st, numSMs, formNu);
}
cudaError_t launch_steps_fp32(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st) {
  return launch_steps_impl<float>(model, P, a, sa, numSMs, st);
}
cudaError_t launch_stages_tma_fp32(int model, int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                  cudaStream_t st) {
  return launch_stages_tma_impl<float>(model, P, a, L, ms, st);
}
}  // namespace selfgpu
