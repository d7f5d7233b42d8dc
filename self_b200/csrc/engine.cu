// The fused tendency engine behind selfgpu_model2d_*: binds the caller's
// (Fortran-owned) device buffers, owns the ping-pong face-trace cache, and
// drives the fused stage kernel through Williamson RK3 steps.  One RK step is
// three launches; after the first step of a given dt the step is replayed from
// a captured CUDA graph.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "fused_stage.cuh"
#include "selfgpu_internal.h"

using namespace selfgpu;

namespace {

// Williamson low-storage RK3, src/SELF_Model.f90:26-29
const double kRK3a[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
const double kRK3g[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

template <int P, class Phys, typename R>
constexpr int elems_per_block() {
  int e = 128 / (P * P);
  if (e < 1) e = 1;
  while (e > 1 && (size_t)e * sizeof(Smem<P, Phys, R>) > 44 * 1024) --e;
  return e;
}

template <int P, class Phys, typename R>
cudaError_t launch_stage(const StageArgs& a, cudaStream_t st) {
  constexpr int EPB = elems_per_block<P, Phys, R>();
  const int grid = (a.nEl + EPB - 1) / EPB;
  k_fused_stage<P, Phys, R, EPB><<<grid, EPB * P * P, 0, st>>>(a);
  return cudaGetLastError();
}

template <class Phys, typename R>
cudaError_t dispatch_P(int P, const StageArgs& a, cudaStream_t st) {
  switch (P) {
    case 2: return launch_stage<2, Phys, R>(a, st);
    case 3: return launch_stage<3, Phys, R>(a, st);
    case 4: return launch_stage<4, Phys, R>(a, st);
    case 5: return launch_stage<5, Phys, R>(a, st);
    case 6: return launch_stage<6, Phys, R>(a, st);
    case 7: return launch_stage<7, Phys, R>(a, st);
    case 8: return launch_stage<8, Phys, R>(a, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
cudaError_t dispatch_model(int model, int P, const StageArgs& a, cudaStream_t st) {
  switch (model) {
    case SELFGPU_MODEL_LSW: return dispatch_P<PhysLSW, R>(P, a, st);
    case SELFGPU_MODEL_SW: return dispatch_P<PhysSW, R>(P, a, st);
    case SELFGPU_MODEL_CIG: return dispatch_P<PhysCIG, R>(P, a, st);
    default: return cudaErrorInvalidValue;
  }
}

__global__ void k_nonfinite(const double* __restrict__ q, long long n, int* flag) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    if (!isfinite(q[k])) {
      atomicExch(flag, 1);
      return;
    }
}

int nt_of(int model) { return model == SELFGPU_MODEL_CIG ? 9 : 3; }
int nv_of(int model) { return model == SELFGPU_MODEL_CIG ? 4 : 3; }

}  // namespace

struct selfgpu_model2d {
  int model = 0, N = 0, P = 0, nEl = 0, form = SELFGPU_FP64;
  cudaStream_t stream = nullptr;
  bool ownStream = false;
  StageArgs base{};
  bool haveInterp = false, haveGeometry = false, haveState = false;
  void* tr[2] = {nullptr, nullptr};
  void* vel[2] = {nullptr, nullptr};
  int cur = 0;     // index of the trace buffer holding the current solution's traces
  int vcur = 0;    // index of the velocity buffer the next stage reads (SW)
  bool valid = false;
  int* dflag = nullptr;
  long long launches = 0;
  // graph cache: one captured RK step per starting buffer parity
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  double graphDt = NAN;

  size_t elemBytes() const { return form == SELFGPU_FP64 ? sizeof(double) : sizeof(float); }

  cudaError_t launch(StageArgs a) {
    ++launches;
    return form == SELFGPU_FP64 ? dispatch_model<double>(model, P, a, stream)
                                : dispatch_model<float>(model, P, a, stream);
  }

  void drop_graphs() {
    for (auto& row : graph)
      for (auto& g : row)
        if (g) {
          cudaGraphExecDestroy(g);
          g = nullptr;
        }
    graphDt = NAN;
  }

  cudaError_t prologue() {
    StageArgs a = base;
    a.mode = MODE_TRACES;
    a.trIn = nullptr;
    a.trOut = tr[cur];
    a.velIn = nullptr;
    a.velOut = (model == SELFGPU_MODEL_SW) ? vel[vcur] : nullptr;
    valid = true;
    return launch(a);
  }

  // Issue the three stages of one RK step starting from the current parities.
  cudaError_t step(double dt) {
    for (int m = 0; m < 3; ++m) {
      StageArgs a = base;
      a.mode = MODE_RK;
      a.rk_a = kRK3a[m];
      a.rk_gdt = kRK3g[m] * dt;
      a.trIn = tr[cur];
      a.trOut = tr[1 - cur];
      if (model == SELFGPU_MODEL_SW) {
        a.velIn = vel[vcur];
        a.velOut = vel[1 - vcur];
        vcur = 1 - vcur;
      }
      cur = 1 - cur;
      cudaError_t e = launch(a);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }
};

static int fail_cuda(const char* where, cudaError_t e) {
  return set_error(SELFGPU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

extern "C" {

int selfgpu_model2d_create(selfgpu_model2d** out, int model, int N, int nEl, int form, void* stream) {
  if (!out) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_create: null handle pointer");
  *out = nullptr;
  if (model != SELFGPU_MODEL_LSW && model != SELFGPU_MODEL_SW && model != SELFGPU_MODEL_CIG)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_create: unknown model id " + std::to_string(model));
  if (N < 1 || N > SELFGPU_MAX_N)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_create: degree N must be in 1.." + std::to_string(SELFGPU_MAX_N));
  if (nEl < 1) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_create: nEl must be >= 1");
  if (form != SELFGPU_FP64 && form != SELFGPU_FP32_BULK)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_create: unknown arithmetic form");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_create", e);
  auto* m = new selfgpu_model2d();
  m->model = model;
  m->N = N;
  m->P = N + 1;
  m->nEl = nEl;
  m->form = form;
  if (stream) {
    m->stream = (cudaStream_t)stream;
  } else {
    // A blocking stream keeps the legacy default-stream ordering of the
    // drop-in API while still allowing graph capture.
    e = cudaStreamCreate(&m->stream);
    if (e != cudaSuccess) {
      delete m;
      return fail_cuda("selfgpu_model2d_create", e);
    }
    m->ownStream = true;
  }
  const size_t trBytes = (size_t)m->P * nt_of(model) * 4 * nEl * m->elemBytes();
  for (int k = 0; k < 2; ++k) {
    e = cudaMalloc(&m->tr[k], trBytes);
    if (e == cudaSuccess && model == SELFGPU_MODEL_SW) e = cudaMalloc(&m->vel[k], (size_t)m->P * 2 * 4 * nEl * m->elemBytes());
    if (e != cudaSuccess) {
      selfgpu_model2d_destroy(m);
      return fail_cuda("selfgpu_model2d_create: trace cache", e);
    }
  }
  e = cudaMalloc(&m->dflag, sizeof(int));
  if (e != cudaSuccess) {
    selfgpu_model2d_destroy(m);
    return fail_cuda("selfgpu_model2d_create", e);
  }
  m->base.nEl = nEl;
  m->base.g = 1.0;
  m->base.gamma = 1.4;
  m->base.Rgas = 1.0;
  *out = m;
  return SELFGPU_OK;
}

int selfgpu_model2d_destroy(selfgpu_model2d* m) {
  if (!m) return SELFGPU_OK;
  if (m->stream) cudaStreamSynchronize(m->stream);
  m->drop_graphs();
  for (int k = 0; k < 2; ++k) {
    if (m->tr[k]) cudaFree(m->tr[k]);
    if (m->vel[k]) cudaFree(m->vel[k]);
  }
  if (m->dflag) cudaFree(m->dflag);
  if (m->ownStream) cudaStreamDestroy(m->stream);
  delete m;
  return SELFGPU_OK;
}

int selfgpu_model2d_set_interp(selfgpu_model2d* m, const double* dgMatrix, const double* bMatrix,
                               const double* qWeights) {
  if (!m || !dgMatrix || !bMatrix || !qWeights) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_interp: null argument");
  const int P = m->P;
  std::memcpy(m->base.dgM, dgMatrix, sizeof(double) * P * P);
  std::memcpy(m->base.bM, bMatrix, sizeof(double) * 2 * P);
  std::memcpy(m->base.qw, qWeights, sizeof(double) * P);
  m->haveInterp = true;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_geometry(selfgpu_model2d* m, const double* dsdx, const double* J, const double* nHat,
                                 const double* nScale, const int* sideInfo_d, const int* sideInfo_h) {
  if (!m || !dsdx || !J || !nHat || !nScale || !sideInfo_d || !sideInfo_h)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_geometry: null argument");
  if (((uintptr_t)dsdx % 16) || ((uintptr_t)nHat % 16))
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_geometry: dsdx and nHat must be 16-byte aligned");
  int rc = validate_side_info(sideInfo_h, m->nEl);
  if (rc != SELFGPU_OK) return rc;
  m->base.dsdx = dsdx;
  m->base.J = J;
  m->base.nHat = nHat;
  m->base.nScale = nScale;
  m->base.sideInfo = sideInfo_d;
  m->haveGeometry = true;
  m->valid = false;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_state(selfgpu_model2d* m, double* solution, double* workSol) {
  if (!m || !solution || !workSol) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_state: null argument");
  m->base.q = solution;
  m->base.G = workSol;
  m->haveState = true;
  m->valid = false;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_field(selfgpu_model2d* m, const char* name, const double* ptr) {
  if (!m || !name) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_field: null argument");
  const std::string n(name);
  int slot = -1;
  if (m->model == SELFGPU_MODEL_LSW) {
    if (n == "H") slot = 0;
    else if (n == "H.boundary") slot = 1;
    else if (n == "fCori") slot = 2;
  } else if (m->model == SELFGPU_MODEL_SW) {
    if (n == "topography.boundary") slot = 0;
    else if (n == "gradTopography") slot = 1;
  } else {
    if (n == "environmentalsGradient") slot = 0;
    else if (n == "environmentals") slot = 1;
    else if (n == "prescribedSolution.boundary") slot = 2;
    else if (n == "prescribedPrimitive.boundary") slot = 3;
    else if (n == "prescribedDiagnostics.boundary") slot = 4;
  }
  if (slot < 0) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_field: unknown field '" + n + "' for this model");
  m->base.fld[slot] = ptr;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_params(selfgpu_model2d* m, double g, double fCori, double expansionFactor, double R) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_params: null handle");
  m->base.g = g;
  m->base.fC = fCori;
  m->base.gamma = expansionFactor;
  m->base.Rgas = R;
  m->valid = false;  // CIG traces depend on gamma
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_invalidate(selfgpu_model2d* m) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_invalidate: null handle");
  m->valid = false;
  return SELFGPU_OK;
}

static int check_ready(selfgpu_model2d* m, const char* where) {
  if (!m) return set_error(SELFGPU_ERR_ARG, std::string(where) + ": null handle");
  if (!m->haveInterp || !m->haveGeometry || !m->haveState)
    return set_error(SELFGPU_ERR_STATE, std::string(where) + ": interp, geometry and state must be set first");
  if (m->model == SELFGPU_MODEL_LSW && (!m->base.fld[0] || !m->base.fld[1]))
    return set_error(SELFGPU_ERR_STATE, std::string(where) + ": LinearShallowWater needs H and H.boundary");
  return SELFGPU_OK;
}

int selfgpu_model2d_tendency(selfgpu_model2d* m, double* dSdt) {
  int rc = check_ready(m, "selfgpu_model2d_tendency");
  if (rc) return rc;
  if (!dSdt) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_tendency: null dSdt");
  cudaError_t e = cudaSuccess;
  if (!m->valid) e = m->prologue();
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_tendency", e);
  StageArgs a = m->base;
  a.mode = MODE_TENDENCY;
  a.dSdt = dSdt;
  a.trIn = m->tr[m->cur];
  a.trOut = nullptr;
  if (m->model == SELFGPU_MODEL_SW) {
    a.velIn = m->vel[m->vcur];
    a.velOut = m->vel[1 - m->vcur];
    m->vcur = 1 - m->vcur;
  }
  e = m->launch(a);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_tendency", e);
  return SELFGPU_OK;
}

int selfgpu_model2d_rk3(selfgpu_model2d* m, double dt, int nSteps) {
  int rc = check_ready(m, "selfgpu_model2d_rk3");
  if (rc) return rc;
  if (nSteps < 0) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_rk3: nSteps < 0");
  cudaError_t e = cudaSuccess;
  if (!m->valid) {
    e = m->prologue();
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_rk3", e);
  }
  if (!(dt == m->graphDt)) m->drop_graphs();
  for (int s = 0; s < nSteps; ++s) {
    cudaGraphExec_t& g = m->graph[m->cur][m->vcur];
    if (s == 0 || g == nullptr) {
      if (g == nullptr && s > 0) {
        // capture one step from this parity
        const int c0 = m->cur, v0 = m->vcur;
        cudaGraph_t graph = nullptr;
        e = cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
          const long long l0 = m->launches;
          e = m->step(dt);
          m->launches = l0;
          cudaError_t e2 = cudaStreamEndCapture(m->stream, &graph);
          if (e == cudaSuccess) e = e2;
        }
        m->cur = c0;
        m->vcur = v0;
        if (e == cudaSuccess) e = cudaGraphInstantiate(&g, graph, 0);
        if (graph) cudaGraphDestroy(graph);
        if (e != cudaSuccess) {
          cudaGetLastError();
          g = nullptr;
        } else {
          m->graphDt = dt;
        }
      }
      if (g == nullptr) {
        e = m->step(dt);
        if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_rk3", e);
        continue;
      }
    }
    e = cudaGraphLaunch(g, m->stream);
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_rk3: graph launch", e);
    m->launches += 3;
    m->cur = 1 - m->cur;  // three swaps per step
    if (m->model == SELFGPU_MODEL_SW) m->vcur = 1 - m->vcur;
  }
  return SELFGPU_OK;
}

int selfgpu_model2d_sync(selfgpu_model2d* m) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_sync: null handle");
  cudaError_t e = cudaStreamSynchronize(m->stream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_sync", e);
  return SELFGPU_OK;
}

int selfgpu_model2d_check_finite(selfgpu_model2d* m) {
  if (!m || !m->haveState) return set_error(SELFGPU_ERR_STATE, "selfgpu_model2d_check_finite: no state bound");
  const long long n = (long long)m->P * m->P * nv_of(m->model) * m->nEl;
  cudaMemsetAsync(m->dflag, 0, sizeof(int), m->stream);
  k_nonfinite<<<296, 256, 0, m->stream>>>(m->base.q, n, m->dflag);
  ++m->launches;
  int h = 0;
  cudaMemcpyAsync(&h, m->dflag, sizeof(int), cudaMemcpyDeviceToHost, m->stream);
  cudaError_t e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_check_finite", e);
  if (h) return set_error(SELFGPU_ERR_NONFINITE, "selfgpu_model2d_check_finite: solution holds NaN or Inf");
  return SELFGPU_OK;
}

long long selfgpu_model2d_launch_count(const selfgpu_model2d* m) { return m ? m->launches : 0; }

}  // extern "C"
