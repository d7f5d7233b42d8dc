// Internal declarations shared by the libselfgpu translation units.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>

#include "../../include/selfgpu.h"

namespace selfgpu {

// Records the calling thread's last error (read back by selfgpu_last_error).
int set_error(int code, const std::string& msg);
const char* last_error();

// Host set-up (setup_host.cpp).
void legendre_quadrature(int N, int type, double* x, double* w);
int lagrange_init(int N, int ctrlType, int M, int tgtType, double* ctrl, double* tgt, double* bw,
                  double* qw, double* iM, double* dM, double* dgM, double* bM);
int mesh2d_structured(int nx, int ny, double x0, double x1, double y0, double y1, int perX, int perY,
                      double amp, int bcid, const int* rot, double* nodeCoords, int* globalNodeIDs,
                      int* sideInfo);
// Neighbour ids may reach nNeighbours (= nEl, or nEl + halo elements).
int validate_side_info(const int* sideInfo, int nEl, int nNeighbours);
// T(k,i) = w_i sqrt((2k+1)/2) L_k(x_i): nodal -> orthonormal Legendre modes
void modal_matrix(int N, const double* x, const double* w, double* T);

// Fused stage launches (stage_fp64_prod.cu / stage_fp64.cu / stage_fp32.cu).
struct StageArgs;
struct StageLaunch {
  bool allowTma;   // use the persistent bulk-copy kernel where it applies
  int smemOptin;   // opt-in shared memory per block (bytes)
  int numSMs;
  int maxGroups;   // cap on the persistent kernel's consumer groups (0 = as many as fit)
};
}  // namespace selfgpu

#include <cuda_runtime.h>

namespace selfgpu {
// production FP64 (stage_fp64_prod.cu), reference roundings (stage_fp64.cu), FP32 bulk
cudaError_t launch_stage_fp64(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                              int* usedTma);
cudaError_t launch_stage_fp64_ref(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                                  int* usedTma);
cudaError_t launch_stage_fp32(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                              int* usedTma);
// nSteps RK3 steps in one cooperative launch (k_fused_steps), per form
struct StepsArgs;
cudaError_t launch_steps_fp64(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st);
cudaError_t launch_steps_fp64_ref(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs,
                                  cudaStream_t st);
cudaError_t launch_steps_fp32(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st);
// several RK stages in one cooperative launch of the persistent kernel
// (k_fused_stage_tma<..., true>; cudaErrorNotSupported where it does not apply)
struct TmaSteps;
cudaError_t launch_stages_tma_fp64(int model, int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                   cudaStream_t st);
cudaError_t launch_stages_tma_fp64_ref(int model, int P, const StageArgs& a, const StageLaunch& L,
                                       const TmaSteps& ms, cudaStream_t st);
cudaError_t launch_stages_tma_fp32(int model, int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                   cudaStream_t st);
// Artificial-viscosity closure (av_closure.cuh).
struct AvArgs;
// closure: the viscosity kernel and the viscous-term kernel of one stage
// (formNu = false: the viscous-term kernel only, with the viscosity already formed)
cudaError_t launch_av_prep_fp64(int P, const AvArgs& a, cudaStream_t st, int numSMs, bool formNu = true);
cudaError_t launch_av_prep_fp32(int P, const AvArgs& a, cudaStream_t st, int numSMs, bool formNu = true);
cudaError_t launch_element_size(const double* J, const double* qw, int P, int nEl, double* h, cudaStream_t st);
cudaError_t launch_closure_features(const double* q, int P, int nEl, const AvArgs& a, float* act, float* feat,
                                    cudaStream_t st);
}  // namespace selfgpu
