// Reference-rounding FP64 instantiation of the fused stage kernels (form
// SELFGPU_FP64_REF) and the FP64 closure kernels.  Built with -fmad=false: no
// multiply-add contraction, and divisions and square roots are IEEE correctly
// rounded, so each value is formed with the same roundings as the reference's
// FP64 CPU path evaluated in the same order.
#include "av_closure.cuh"
#include "stage_dispatch.cuh"

namespace selfgpu {
cudaError_t launch_stage_fp64_ref(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                                  int* usedTma) {
  return launch_stage_impl<double>(model, P, a, L, st, usedTma);
}

cudaError_t launch_av_prep_fp64(int P, const AvArgs& a, cudaStream_t st, int numSMs, bool formNu) {
  return launch_av_prep_impl<double>(P, a, st, numSMs, formNu);
}

// h = sqrt(sum_j sum_i w_i w_j J_ij), in the oracle's summation order
__global__ void k_element_size(const double* __restrict__ J, QwArr qw, int P, int nEl, double* __restrict__ h) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nEl; e += (long long)gridDim.x * blockDim.x) {
    double area = 0.0;
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) area = area + qw.w[i] * qw.w[j] * J[i + P * (j + (long long)P * e)];
    h[e] = sqrt(area);
  }
}

cudaError_t launch_element_size(const double* J, const double* qw, int P, int nEl, double* h, cudaStream_t st) {
  QwArr w{};
  for (int k = 0; k < P; ++k) w.w[k] = qw[k];
  k_element_size<<<(nEl + 255) / 256, 256, 0, st>>>(J, w, P, nEl, h);
  return cudaGetLastError();
}

cudaError_t launch_closure_features(const double* q, int P, int nEl, const AvArgs& a, float* act, float* feat,
                                    cudaStream_t st) {
  switch (P) {
#define SG_FEAT_CASE(PV)                                                  \
  case PV:                                                                \
    k_closure_features<PV><<<nEl, PV * PV, 0, st>>>(q, nEl, a, act, feat); \
    return cudaGetLastError();
    SG_FEAT_CASE(2)
    SG_FEAT_CASE(3)
    SG_FEAT_CASE(4)
    SG_FEAT_CASE(5)
    SG_FEAT_CASE(6)
    SG_FEAT_CASE(7)
    SG_FEAT_CASE(8)
#undef SG_FEAT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}
cudaError_t launch_steps_fp64_ref(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st) {
  return launch_steps_impl<double>(model, P, a, sa, numSMs, st);
}
cudaError_t launch_stages_tma_fp64_ref(int model, int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                      cudaStream_t st) {
  return launch_stages_tma_impl<double>(model, P, a, L, ms, st);
}
}  // namespace selfgpu
