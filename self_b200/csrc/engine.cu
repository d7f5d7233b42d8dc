// The fused tendency engine behind selfgpu_model2d_*: binds the caller's
// (Fortran-owned) device buffers, owns the ping-pong face-trace cache, and
// drives the fused stage kernel through Williamson RK3 steps.  One RK step is
// three launches; after the first step of a given dt the step is replayed from
// a captured CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "av_closure.cuh"
#include "fused_stage.cuh"
#include "fused_stage_tma.cuh"
#include "selfgpu_internal.h"

using namespace selfgpu;

namespace {

// Williamson low-storage RK3, src/SELF_Model.f90:26-29
const double kRK3a[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
const double kRK3g[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

__global__ void k_nonfinite(const double* __restrict__ q, long long n, int* flag) {
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    if (!isfinite(q[k])) {
      atomicExch(flag, 1);
      return;
    }
}

// One element's packed geometry record of the given GeoKind (geo_rec(P,
// kind).bytes): dsdx (4 P^2 values, two planes of per-node pairs), nHat (8 P),
// nScale (4 P) -- FP64, or FP32 rounded to nearest in GEO_F32 -- then J
// (GEO_REF) or 1/J (GEO_INVJ, GEO_F32) in FP64, none in GEO_NOJ, then
// sideInfo's 20 ints.  One thread per 32-bit word of the records.
__global__ void k_pack_geometry(const double* __restrict__ dsdx, const double* __restrict__ nHat,
                                const double* __restrict__ nScale, const double* __restrict__ J,
                                const int* __restrict__ sideInfo, int P, int nEl, int kind,
                                uint32_t* __restrict__ out) {
  const GeoRec gr = geo_rec(P, kind);
  const int PP = P * P, words = gr.bytes / 4;
  const long long total = (long long)words * nEl;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const long long e = k / words;
    const int b = 4 * (int)(k - e * words);  // byte offset within the record
    double v = 0.0;
    if (b < gr.oJ) {  // metric terms: value index s
      int s = b / gr.wm;
      if (s < 4 * PP) {  // plane s / (2 P^2), node (s mod 2 P^2) / 2, component s mod 2
        const int pl = s / (2 * PP), r = s - pl * 2 * PP;
        v = dsdx[4 * PP * e + 4 * (r >> 1) + 2 * pl + (r & 1)];
      } else if ((s -= 4 * PP) < 8 * P) {
        v = nHat[8 * P * e + s];
      } else {
        v = nScale[4 * P * e + s - 8 * P];
      }
      if (gr.wm == 4) {
        out[k] = __float_as_uint(__double2float_rn(v));
        continue;
      }
    } else if (b < gr.oSi) {
      const int s = (b - gr.oJ) / 8;
      v = kind == GEO_REF ? J[PP * e + s] : 1.0 / J[PP * e + s];
    } else {
      out[k] = (uint32_t)sideInfo[20 * e + (b - gr.oSi) / 4];
      continue;
    }
    const unsigned long long u = (unsigned long long)__double_as_longlong(v);
    out[k] = (b & 4) ? (uint32_t)(u >> 32) : (uint32_t)u;  // little-endian halves of the double
  }
}

// Gather (scatter = 0) or scatter (scatter = 1) of n cache blocks of `words`
// 32-bit words: packed[k] <-> cache[blocks[k]].
__global__ void k_move_blocks(const uint32_t* __restrict__ src, const int* __restrict__ blocks, int n, int words,
                              uint32_t* __restrict__ dst, int scatter) {
  const long long total = (long long)n * words;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const long long b = k / words, w = k - b * words;
    const long long c = (long long)blocks[b] * words + w;
    if (scatter) dst[c] = src[k];
    else dst[k] = src[c];
  }
}

// Entropy integrands (CalculateEntropy of the three models), summed per
// element in the reference's node order (j outer, i inner):
//   LSW  0.5 (H (u^2 + v^2) + g eta^2) J w_i w_j  (src/models/SELF_LinearShallowWater.f90:171-216)
//   SW   (0.5 (Hu^2/H + Hv^2/H) + 0.5 g H^2 - g H b) J w_i w_j  (src/models/SELF_ShallowWater.f90:149-188)
//   CIG  rho (log p - gamma log rho) / (gamma - 1) w_i w_j J, p from the
//        solution as ConservativeToPrimitive forms it (src/models/SELF_CompressibleIdealGas2D.f90:782-823)
// `aux` is H (LSW) or the topography b (SW), (P,P,1,nEl).
__global__ void k_entropy_elements(int model, const double* __restrict__ q, const double* __restrict__ J,
                                   const double* __restrict__ aux, QwArr qw, int P, int nEl, double g, double gamma,
                                   double* __restrict__ out) {
  const int PP = P * P;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nEl; e += (long long)gridDim.x * blockDim.x) {
    const int nv = model == SELFGPU_MODEL_CIG ? 4 : 3;
    const double* qe = q + (size_t)nv * PP * e;
    double s = 0.0;
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) {
        const int n = i + P * j;
        const double Jac = J[n + (size_t)PP * e], wi = qw.w[i], wj = qw.w[j];
        if (model == SELFGPU_MODEL_LSW) {
          const double u = qe[n], v = qe[n + PP], eta = qe[n + 2 * PP], H = aux[n + (size_t)PP * e];
          s = s + 0.5 * (H * (u * u + v * v) + g * eta * eta) * Jac * wi * wj;
        } else if (model == SELFGPU_MODEL_SW) {
          const double Hu = qe[n], Hv = qe[n + PP], H = qe[n + 2 * PP];
          const double b = aux ? aux[n + (size_t)PP * e] : 0.0;
          s = s + (0.5 * (Hu * Hu / H + Hv * Hv / H) + 0.5 * g * H * H - g * H * b) * Jac * wi * wj;
        } else {
          const double rhoU = qe[n], rhoV = qe[n + PP], rho = qe[n + 2 * PP], rhoE = qe[n + 3 * PP];
          const double u = rhoU / rho, v = rhoV / rho;
          const double p = (gamma - 1.0) * (rhoE - 0.5 * (rhoU * u + rhoV * v));
          s = s + rho * (log(p) - gamma * log(rho)) / (gamma - 1.0) * wi * wj * Jac;
        }
      }
    out[e] = s;
  }
}

// Deterministic sum of n values by one block: strided partial sums, then a
// shared-memory tree.  The result lands in out[0].
__global__ void __launch_bounds__(1024) k_sum_block(const double* __restrict__ x, long long n, double* out) {
  __shared__ double part[1024];
  double s = 0.0;
  for (long long k = threadIdx.x; k < n; k += blockDim.x) s += x[k];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = part[0];
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
  int nHalo = 0;   // halo elements after the rank's own in the caches (multi-rank runs)
  int cur = 0;     // index of the trace buffer holding the current solution's traces
  int vcur = 0;    // index of the velocity buffer the next stage reads (SW)
  bool valid = false;
  int* dflag = nullptr;
  int* derr = nullptr;  // error word of the persistent kernel's bounded waits
  long long launches = 0;
  long long tmaLaunches = 0;
  StageLaunch cfg{true, 0, 148, 0};
  // graph cache: one captured RK step per starting buffer parity
  cudaGraphExec_t graph[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  long long graphTma[2][2] = {{0, 0}, {0, 0}};
  long long graphLaunches[2][2] = {{0, 0}, {0, 0}};
  double graphDt = NAN;
  // artificial-viscosity closure (CIG): mode, per-launch arguments and buffers
  int avMode = AV_OFF;
  AvArgs av{};
  double* avNu = nullptr;
  float* avAct = nullptr;  // [0, nEl): activation applied, [nEl, 2 nEl): indicator activation
  int* avFallbacks = nullptr;  // [0] MLP fallbacks, [1] MLP evaluations, [2] active count, then the active list
  double* avH = nullptr;
  void* avVisc = nullptr;
  void* avVtr = nullptr;
  __nv_bfloat16* mlpW = nullptr;
  float* mlpB = nullptr;
  double* geo = nullptr;  // packed geometry records (persistent kernel)
  float* gf = nullptr;    // RK register of the FP32-bulk form (P,P,NV,nEl); workSol is unused then
  double* entropyBuf = nullptr;  // per-element entropy sums (nEl) and the total
  bool multistep = false;         // rk3 as one cooperative launch where the mesh fits one wave
  bool multistage = false;        // rk3 as one launch of the persistent kernel over all stages
  unsigned* stepBar = nullptr;    // grid-barrier / stage-end counter of the one-launch paths

  size_t elemBytes() const { return form == SELFGPU_FP32_BULK ? sizeof(float) : sizeof(double); }

  // stage kernels of this handle's arithmetic form
  static cudaError_t launch_stage_form(int form, int model, int P, const StageArgs& a, const StageLaunch& L,
                                       cudaStream_t st, int* usedTma) {
    switch (form) {
      case SELFGPU_FP64: return launch_stage_fp64(model, P, a, L, st, usedTma);
      case SELFGPU_FP64_REF: return launch_stage_fp64_ref(model, P, a, L, st, usedTma);
      default: return launch_stage_fp32(model, P, a, L, st, usedTma);
    }
  }

  // closure preparation of one stage: element viscosity (formNu: the first
  // stage of an RK step and tendency evaluations; the step's other stages
  // keep it), BR1 gradient, viscous volume flux and traces, from the
  // solution and the trace cache trIn
  cudaError_t launch_av(const void* trIn, bool formNu = true) {
    AvArgs x = av;
    x.nEl = nEl;
    x.q = base.q;
    x.dsdx = base.dsdx;
    x.J = base.J;
    x.nHat = base.nHat;
    x.nScale = base.nScale;
    x.sideInfo = base.sideInfo;
    x.trIn = trIn;
    x.presc = base.fld[2];
    x.gamma = base.gamma;
    launches += formNu ? 2 : 1;
    return form == SELFGPU_FP32_BULK ? launch_av_prep_fp32(P, x, stream, cfg.numSMs, formNu)
                                     : launch_av_prep_fp64(P, x, stream, cfg.numSMs, formNu);
  }

  cudaError_t launch(StageArgs a, bool formNu = true) {
    if (avMode != AV_OFF && a.mode != MODE_TRACES) {
      cudaError_t e = launch_av(a.trIn, formNu);
      if (e != cudaSuccess) return e;
    }
    ++launches;
    int tma = 0;
    cudaError_t e = launch_stage_form(form, model, P, a, cfg, stream, &tma);
    tmaLaunches += tma;
    return e;
  }

  // nSteps RK3 steps as one cooperative launch of k_fused_steps from the
  // current parities; cudaErrorCooperativeLaunchTooLarge when the element
  // groups do not fit one wave of resident CTAs (the caller falls back).
  cudaError_t launch_steps(double dt, int nSteps) {
    cudaError_t e = cudaSuccess;
    if (!stepBar) e = cudaMalloc(&stepBar, sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(stepBar, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    StepsArgs sa{};
    sa.nSteps = nSteps;
    sa.dt = dt;
    for (int k = 0; k < 3; ++k) {
      sa.rkA[k] = kRK3a[k];
      sa.rkG[k] = kRK3g[k];
    }
    sa.tr[0] = tr[0];
    sa.tr[1] = tr[1];
    sa.vel[0] = vel[0];
    sa.vel[1] = vel[1];
    sa.cur = cur;
    sa.vcur = vcur;
    sa.bar = stepBar;
    StageArgs a = base;
    a.mode = MODE_RK;
    switch (form) {
      case SELFGPU_FP64: e = launch_steps_fp64(model, P, a, sa, cfg.numSMs, stream); break;
      case SELFGPU_FP64_REF: e = launch_steps_fp64_ref(model, P, a, sa, cfg.numSMs, stream); break;
      default: e = launch_steps_fp32(model, P, a, sa, cfg.numSMs, stream); break;
    }
    if (e != cudaSuccess) return e;
    ++launches;
    if ((3LL * nSteps) & 1) {  // three cache swaps per step
      cur = 1 - cur;
      if (model == SELFGPU_MODEL_SW) vcur = 1 - vcur;
    }
    return cudaSuccess;
  }

  unsigned long long gen = 0;  // bumped whenever captured work goes stale (ensemble graphs check it)

  // nSteps RK3 steps as launches of the persistent kernel that each run many
  // stages (k_fused_stage_tma<..., true>), from the current parities;
  // cudaErrorNotSupported / cudaErrorCooperativeLaunchTooLarge when that
  // kernel does not apply (the caller falls back).
  cudaError_t launch_stages_tma(double dt, int nSteps) {
    cudaError_t e = cudaSuccess;
    if (!stepBar) e = cudaMalloc(&stepBar, sizeof(unsigned));
    if (e != cudaSuccess) return e;
    StageArgs a = base;
    a.mode = MODE_RK;
    constexpr int kChunk = 100000;  // steps per launch: the stage-end counter stays below 2^32
    for (int done = 0; done < nSteps;) {
      const int n = (nSteps - done) < kChunk ? (nSteps - done) : kChunk;
      e = cudaMemsetAsync(stepBar, 0, sizeof(unsigned), stream);
      if (e != cudaSuccess) return e;
      TmaSteps ms{};
      ms.nStages = 3 * n;
      ms.dt = dt;
      for (int k = 0; k < 3; ++k) {
        ms.rkA[k] = kRK3a[k];
        ms.rkG[k] = kRK3g[k];
      }
      ms.tr[0] = tr[0];
      ms.tr[1] = tr[1];
      ms.vel[0] = vel[0];
      ms.vel[1] = vel[1];
      ms.cur0 = cur;
      ms.vcur0 = vcur;
      ms.bar = stepBar;
      switch (form) {
        case SELFGPU_FP64: e = launch_stages_tma_fp64(model, P, a, cfg, ms, stream); break;
        case SELFGPU_FP64_REF: e = launch_stages_tma_fp64_ref(model, P, a, cfg, ms, stream); break;
        default: e = launch_stages_tma_fp32(model, P, a, cfg, ms, stream); break;
      }
      if (e != cudaSuccess) return e;
      ++launches;
      ++tmaLaunches;
      if ((3LL * n) & 1) {  // three cache swaps per step
        cur = 1 - cur;
        if (model == SELFGPU_MODEL_SW) vcur = 1 - vcur;
      }
      done += n;
    }
    return cudaSuccess;
  }

  void drop_graphs() {
    ++gen;
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

  // Issue RK stage m (0, 1, 2) from the current parities.
  cudaError_t stage_once(double dt, int m) {
    StageArgs a = base;
    a.mode = MODE_RK;
    a.rk_a = kRK3a[m];
    a.rk_gdt = kRK3g[m] * dt;
    a.rk_g = kRK3g[m];
    a.trIn = tr[cur];
    a.trOut = tr[1 - cur];
    if (model == SELFGPU_MODEL_SW) {
      a.velIn = vel[vcur];
      a.velOut = vel[1 - vcur];
      vcur = 1 - vcur;
    }
    cur = 1 - cur;
    return launch(a, m == 0);  // the closure's viscosity: once per RK step, from the step's first stage
  }

  // Issue the three stages of one RK step starting from the current parities.
  cudaError_t step(double dt) {
    for (int m = 0; m < 3; ++m) {
      cudaError_t e = stage_once(dt, m);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  }

  size_t trace_block_bytes() const {  // one (element, side) block of the trace cache
    const size_t per16 = 16 / elemBytes();
    return ((size_t)nt_of(model) * P + per16 - 1) / per16 * per16 * elemBytes();
  }
  size_t vel_block_bytes() const { return (size_t)2 * P * elemBytes(); }

  cudaError_t alloc_caches() {
    for (int k = 0; k < 2; ++k) {
      if (tr[k]) cudaFree(tr[k]);
      if (vel[k]) cudaFree(vel[k]);
      tr[k] = vel[k] = nullptr;
    }
    const size_t nb = 4 * (size_t)(nEl + nHalo);
    for (int k = 0; k < 2; ++k) {
      cudaError_t e = cudaMalloc(&tr[k], trace_block_bytes() * nb);
      if (e == cudaSuccess && model == SELFGPU_MODEL_SW) e = cudaMalloc(&vel[k], vel_block_bytes() * nb);
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
  if (form != SELFGPU_FP64 && form != SELFGPU_FP64_REF && form != SELFGPU_FP32_BULK)
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
  // all stages of an rk3 call in one launch where that applies (N = 7, meshes
  // of 4 440 to 35 520 elements; 5 328 to 42 624 with twelve groups, 6 216 to 49 728 with fourteen): measured 1-4 % faster per stage in these
  // forms, and slower for some models in the reference-rounding form, which
  // keeps stage launches
  m->multistage = form != SELFGPU_FP64_REF;
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
  // one (element, side) block holds NT fields x P nodes, padded to 16 bytes
  // (trace_side_stride in fused_stage.cuh)
  e = m->alloc_caches();
  if (e != cudaSuccess) {
    selfgpu_model2d_destroy(m);
    return fail_cuda("selfgpu_model2d_create: trace cache", e);
  }
  e = cudaMalloc(&m->dflag, 2 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(m->dflag, 0, 2 * sizeof(int));
  if (e != cudaSuccess) {
    selfgpu_model2d_destroy(m);
    return fail_cuda("selfgpu_model2d_create", e);
  }
  m->derr = m->dflag + 1;
  cudaDeviceGetAttribute(&m->cfg.smemOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&m->cfg.numSMs, cudaDevAttrMultiProcessorCount, dev);
  m->base.err = m->derr;
  m->base.waitCycles = 4000000000LL;  // about 2 s at the B200 boost clock
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
  for (void* p : {(void*)m->avNu, (void*)m->avAct, (void*)m->avFallbacks, (void*)m->avH, m->avVisc, m->avVtr,
                  (void*)m->mlpW, (void*)m->mlpB, (void*)m->geo, (void*)m->entropyBuf, (void*)m->stepBar,
                  (void*)m->gf})
    if (p) cudaFree(p);
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
  for (int k = 0; k < 2 * P; ++k) m->base.bMf[k] = (float)bMatrix[k];
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
  int rc = validate_side_info(sideInfo_h, m->nEl, m->nEl + m->nHalo);
  if (rc != SELFGPU_OK) return rc;
  m->base.dsdx = dsdx;
  m->base.J = J;
  m->base.nHat = nHat;
  m->base.nScale = nScale;
  m->base.sideInfo = sideInfo_d;
  // Packed per-element geometry records for the persistent kernel, built on
  // the legacy default stream after whatever produced the arrays, and waited
  // for (set-up time): the caller's arrays stay the source of truth, and a
  // caller that changes them calls set_geometry again.
  const int P = m->P;
  // the record kind the form's stage kernel reads (geo_kind)
  const int kind = m->form == SELFGPU_FP32_BULK ? GEO_F32
                   : m->form == SELFGPU_FP64_REF ? GEO_REF
                   : (P == 8 ? GEO_NOJ : GEO_INVJ);
  const GeoRec gr = geo_rec(P, kind);
  cudaError_t e = cudaSuccess;
  if (!m->geo) e = cudaMalloc(&m->geo, (size_t)gr.bytes * m->nEl);
  if (e == cudaSuccess) {
    const long long total = (long long)(gr.bytes / 4) * m->nEl;
    const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    k_pack_geometry<<<blocks, 256, 0, 0>>>(dsdx, nHat, nScale, J, sideInfo_d, P, m->nEl, kind,
                                           reinterpret_cast<uint32_t*>(m->geo));
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(0);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_set_geometry", e);
  m->base.geo = m->geo;
  m->haveGeometry = true;
  m->valid = false;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_state(selfgpu_model2d* m, double* solution, double* workSol) {
  if (!m || !solution || !workSol) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_state: null argument");
  m->base.q = solution;
  m->base.G = workSol;
  if (m->form == SELFGPU_FP32_BULK && !m->gf) {
    // the FP32-bulk form keeps its RK register in FP32, in engine memory
    const size_t n = (size_t)m->P * m->P * nv_of(m->model) * m->nEl;
    cudaError_t e = cudaMalloc(&m->gf, n * sizeof(float));
    if (e == cudaSuccess) e = cudaMemsetAsync(m->gf, 0, n * sizeof(float), m->stream);
    if (e != cudaSuccess) {
      if (m->gf) cudaFree(m->gf);
      m->gf = nullptr;
      return fail_cuda("selfgpu_model2d_set_state", e);
    }
    m->base.Gf = m->gf;
  }
  m->haveState = true;
  m->valid = false;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_field(selfgpu_model2d* m, const char* name, const double* ptr) {
  if (!m || !name) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_field: null argument");
  const std::string n(name);
  if (n == "elementDt") {  // per-element time step (nEl doubles); replaces dt in selfgpu_model2d_rk3
    m->base.dtElem = ptr;
    m->drop_graphs();
    return SELFGPU_OK;
  }
  int slot = -1;
  if (m->model == SELFGPU_MODEL_LSW) {
    if (n == "H") slot = 0;
    else if (n == "H.boundary") slot = 1;
    else if (n == "fCori") slot = 2;
  } else if (m->model == SELFGPU_MODEL_SW) {
    if (n == "topography.boundary") slot = 0;
    else if (n == "gradTopography") slot = 1;
    else if (n == "topography") slot = 2;  // interior topography: read by the entropy only
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
  if (m->gf) {  // a new state: the FP32-bulk form's RK register starts from zero (as a zeroed workSol would)
    const size_t n = (size_t)m->P * m->P * nv_of(m->model) * m->nEl;
    cudaError_t e = cudaMemsetAsync(m->gf, 0, n * sizeof(float), m->stream);
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_invalidate", e);
  }
  return SELFGPU_OK;
}

static int check_ready(selfgpu_model2d* m, const char* where) {
  if (!m) return set_error(SELFGPU_ERR_ARG, std::string(where) + ": null handle");
  if (!m->haveInterp || !m->haveGeometry || !m->haveState)
    return set_error(SELFGPU_ERR_STATE, std::string(where) + ": interp, geometry and state must be set first");
  if (m->model == SELFGPU_MODEL_LSW && (!m->base.fld[0] || !m->base.fld[1]))
    return set_error(SELFGPU_ERR_STATE, std::string(where) + ": LinearShallowWater needs H and H.boundary");
  if (m->model == SELFGPU_MODEL_CIG) {
    const int np = (m->base.fld[2] != nullptr) + (m->base.fld[3] != nullptr) + (m->base.fld[4] != nullptr);
    if (np != 0 && np != 3)
      return set_error(SELFGPU_ERR_STATE, std::string(where) +
                                              ": set all three prescribed boundary fields or none of them");
  }
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
  if (m->multistage && nSteps > 0 && m->avMode == AV_OFF && m->nHalo == 0 && m->base.debugStarve != 1 &&
      m->cfg.allowTma) {
    e = m->valid ? cudaSuccess : m->prologue();
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_rk3", e);
    const int c0 = m->cur, v0 = m->vcur;
    e = m->launch_stages_tma(dt, nSteps);
    if (e == cudaSuccess) return SELFGPU_OK;
    cudaGetLastError();
    if (e != cudaErrorNotSupported && e != cudaErrorCooperativeLaunchTooLarge)
      return fail_cuda("selfgpu_model2d_rk3: multi-stage launch", e);
    m->cur = c0;  // nothing was launched: stage launches below
    m->vcur = v0;
  }
  if (m->multistep && nSteps > 0 && m->avMode == AV_OFF && m->nHalo == 0 && !m->base.debugStarve) {
    e = m->valid ? cudaSuccess : m->prologue();
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_rk3", e);
    e = m->launch_steps(dt, nSteps);
    if (e == cudaSuccess) return SELFGPU_OK;
    cudaGetLastError();
    if (e != cudaErrorCooperativeLaunchTooLarge) return fail_cuda("selfgpu_model2d_rk3: multi-step launch", e);
    // the mesh does not fit one wave: graph-replayed steps below
  }
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
          const long long l0 = m->launches, t0 = m->tmaLaunches;
          e = m->step(dt);
          m->graphTma[c0][v0] = m->tmaLaunches - t0;
          m->graphLaunches[c0][v0] = m->launches - l0;
          m->launches = l0;
          m->tmaLaunches = t0;
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
    m->launches += m->graphLaunches[m->cur][m->vcur];
    m->tmaLaunches += m->graphTma[m->cur][m->vcur];
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
  int werr = 0;
  e = cudaMemcpy(&werr, m->derr, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_sync", e);
  if (werr) {
    cudaMemset(m->derr, 0, sizeof(int));
    m->valid = false;
    return set_error(SELFGPU_ERR_TIMEOUT,
                     "selfgpu_model2d_sync: a bounded device wait ran out; the solution of this call is invalid");
  }
  return SELFGPU_OK;
}

int selfgpu_model2d_set_wait_limit(selfgpu_model2d* m, long long cycles) {
  if (!m || cycles < 1000) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_wait_limit: bad arguments");
  m->base.waitCycles = cycles;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_inject_stall(selfgpu_model2d* m, int enable) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_inject_stall: null handle");
  if (enable < 0 || enable > 2) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_inject_stall: enable is 0, 1 or 2");
  m->base.debugStarve = enable;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_multistep(selfgpu_model2d* m, int enable) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_multistep: null handle");
  m->multistep = enable != 0;
  return SELFGPU_OK;
}

int selfgpu_model2d_set_kernel(selfgpu_model2d* m, int persistent) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_kernel: null handle");
  m->cfg.allowTma = persistent != 0;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_multistage(selfgpu_model2d* m, int enable) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_multistage: null handle");
  m->multistage = enable != 0;
  return SELFGPU_OK;
}

int selfgpu_model2d_set_launch(selfgpu_model2d* m, int persistent, int groups) {
  if (!m || groups < 0) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_launch: bad arguments");
  m->cfg.allowTma = persistent != 0;
  m->cfg.maxGroups = groups;
  m->drop_graphs();
  return SELFGPU_OK;
}

long long selfgpu_model2d_persistent_launch_count(const selfgpu_model2d* m) { return m ? m->tmaLaunches : 0; }

int selfgpu_model2d_autotune(selfgpu_model2d* m, int* persistent, int* groups, float* usPerStage) {
  int rc = check_ready(m, "selfgpu_model2d_autotune");
  if (rc) return rc;
  // Candidates: the per-element-group kernel and the persistent kernel with
  // every consumer-group count from 2 up to what fits.  Each is timed on
  // RK-stage launches over scratch copies of the solution and RK register
  // (a zero step: the state is not modified); the stage writes the trace
  // caches the next real stage rewrites anyway.
  const size_t n = (size_t)m->P * m->P * nv_of(m->model) * m->nEl;
  double* scratch = nullptr;
  cudaError_t e = cudaMalloc(&scratch, 2 * n * sizeof(double));
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_autotune", e);
  e = cudaMemcpyAsync(scratch, m->base.q, n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
  if (e == cudaSuccess) {
    if (m->gf)  // the FP32-bulk form's register (n floats fit the second half)
      e = cudaMemcpyAsync(scratch + n, m->gf, n * sizeof(float), cudaMemcpyDeviceToDevice, m->stream);
    else
      e = cudaMemcpyAsync(scratch + n, m->base.G, n * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
  }
  if (e != cudaSuccess) {
    cudaFree(scratch);
    return fail_cuda("selfgpu_model2d_autotune", e);
  }
  if (!m->valid) {
    e = m->prologue();
    if (e != cudaSuccess) {
      cudaFree(scratch);
      return fail_cuda("selfgpu_model2d_autotune", e);
    }
  }
  StageArgs a = m->base;
  a.mode = MODE_RK;
  a.q = scratch;
  a.G = scratch + n;
  if (m->gf) a.Gf = reinterpret_cast<float*>(scratch + n);
  a.rk_a = 0.0;
  a.rk_gdt = 0.0;
  a.rk_g = 0.0;
  a.trIn = m->tr[m->cur];
  a.trOut = m->tr[1 - m->cur];  // rewritten by the next real stage
  if (m->model == SELFGPU_MODEL_SW) {
    a.velIn = m->vel[m->vcur];
    a.velOut = m->vel[1 - m->vcur];  // likewise; the cache parity is left unchanged
  }
  if (m->avMode != AV_OFF) {
    e = m->launch_av(a.trIn);  // the candidates then read this state's viscous terms
    if (e != cudaSuccess) {
      cudaFree(scratch);
      return fail_cuda("selfgpu_model2d_autotune", e);
    }
  }
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const StageLaunch saved = m->cfg;
  float best = 1e30f;
  StageLaunch bestCfg = saved;
  // consumer groups per CTA: up to 10 two-warp groups for P >= 6 (at P = 8, 14
  // in the FP32-bulk form, 12 for the production FP64 ShallowWater models), up
  // to 20 one-warp groups for P <= 4, 24 in FP32 (TmaTraits::kMaxGroups)
  const bool twelve = m->P == 8 && (m->form == SELFGPU_FP32_BULK ||
                                    (m->form == SELFGPU_FP64 && m->model != SELFGPU_MODEL_CIG));
  const int maxCand = m->P <= 4 ? (m->form == SELFGPU_FP32_BULK ? 23 : 19)
                                  : (m->form == SELFGPU_FP32_BULK && m->P == 8 ? 13 : twelve ? 11 : 9);
  for (int cand = 0; cand <= maxCand; ++cand) {
    StageLaunch c = saved;
    if (cand == 0) {
      c.allowTma = false;
    } else {
      c.allowTma = true;
      c.maxGroups = cand + 1;  // capped by what fits in shared memory
    }
    m->cfg = c;
    int tma = 0;
    e = selfgpu_model2d::launch_stage_form(m->form, m->model, m->P, a, c, m->stream, &tma);
    if (e != cudaSuccess) break;
    if (cand > 0 && !tma) break;  // the persistent kernel does not apply
    cudaEventRecord(t0, m->stream);
    for (int r = 0; r < 3; ++r)
      selfgpu_model2d::launch_stage_form(m->form, m->model, m->P, a, c, m->stream, &tma);
    cudaEventRecord(t1, m->stream);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    if (ms < best) {
      best = ms;
      bestCfg = c;
    }
  }
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(scratch);
  if (e != cudaSuccess) {
    m->cfg = saved;
    return fail_cuda("selfgpu_model2d_autotune", e);
  }
  m->cfg = bestCfg;
  m->drop_graphs();
  if (persistent) *persistent = bestCfg.allowTma ? 1 : 0;
  if (groups) *groups = bestCfg.allowTma ? bestCfg.maxGroups : 0;
  if (usPerStage) *usPerStage = best * 1000.f / 3.f;
  return SELFGPU_OK;
}

int selfgpu_model2d_set_closure(selfgpu_model2d* m, int mode, double c, double s0, double kappa,
                                const double* controlPoints) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_closure: null handle");
  if (mode == AV_OFF) {
    m->avMode = AV_OFF;
    m->base.av = 0;
    m->drop_graphs();
    return SELFGPU_OK;
  }
  if (m->model != SELFGPU_MODEL_CIG)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_closure: the closure is defined for CompressibleIdealGas2D");
  if (m->nHalo > 0)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_closure: the closure is single-rank (no halo exchange of "
                                      "viscous terms)");
  if (mode != AV_INDICATOR && mode != AV_MLP)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_closure: unknown closure mode");
  if (mode == AV_MLP && (m->P < 6 || !m->mlpW))
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_closure: the MLP closure needs N >= 5 and weights "
                                      "(selfgpu_model2d_set_mlp)");
  if (!controlPoints || !(kappa > 0.0) || !(c >= 0.0))
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_closure: bad arguments");
  if (!m->haveInterp || !m->haveGeometry)
    return set_error(SELFGPU_ERR_STATE, "selfgpu_model2d_set_closure: interp and geometry must be set first");
  const size_t nEl = (size_t)m->nEl, PP = (size_t)m->P * m->P;
  cudaError_t e = cudaSuccess;
  if (!m->avNu) {
    e = cudaMalloc(&m->avNu, nEl * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&m->avAct, 2 * nEl * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->avFallbacks, (3 + nEl) * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&m->avH, nEl * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&m->avVisc, 8 * PP * nEl * m->elemBytes());
    if (e == cudaSuccess) e = cudaMalloc(&m->avVtr, 4 * 8 * (size_t)m->P * nEl * m->elemBytes());
    if (e == cudaSuccess) e = cudaMemsetAsync(m->avFallbacks, 0, 2 * sizeof(int), m->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(m->avAct, 0, 2 * nEl * sizeof(float), m->stream);
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_set_closure", e);
  }
  AvArgs& x = m->av;
  x.mode = mode;
  x.avC = c;
  x.s0 = s0;
  x.kappa = kappa;
  modal_matrix(m->N, controlPoints, m->base.qw, x.T);
  std::memcpy(x.dgM, m->base.dgM, sizeof(x.dgM));
  std::memcpy(x.bM, m->base.bM, sizeof(x.bM));
  std::memcpy(x.qw, m->base.qw, sizeof(x.qw));
  x.hEl = m->avH;
  x.nu = m->avNu;
  x.act = m->avAct;
  x.actInd = m->avAct + nEl;
  x.fallbacks = m->avFallbacks;
  x.activeCount = m->avFallbacks + 2;
  x.activeList = m->avFallbacks + 3;
  x.visc = m->avVisc;
  x.vtr = m->avVtr;
  x.mlpW = m->mlpW;
  x.mlpB = m->mlpB;
  e = launch_element_size(m->base.J, m->base.qw, m->P, m->nEl, m->avH, m->stream);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_set_closure", e);
  m->avMode = mode;
  m->base.av = 1;
  m->base.visc = m->avVisc;
  m->base.vtr = m->avVtr;
  m->base.avNu = m->avNu;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_set_mlp(selfgpu_model2d* m, const uint16_t* weights, const float* params) {
  if (!m || !weights || !params) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_mlp: null argument");
  cudaError_t e = cudaSuccess;
  if (!m->mlpW) {
    e = cudaMalloc(&m->mlpW, kMlpWeights * sizeof(__nv_bfloat16));
    if (e == cudaSuccess) e = cudaMalloc(&m->mlpB, kMlpFloats * sizeof(float));
    if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_set_mlp", e);
  }
  e = cudaMemcpyAsync(m->mlpW, weights, kMlpWeights * sizeof(uint16_t), cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(m->mlpB, params, kMlpFloats * sizeof(float), cudaMemcpyHostToDevice, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_set_mlp", e);
  m->av.mlpW = m->mlpW;
  m->av.mlpB = m->mlpB;
  m->drop_graphs();
  return SELFGPU_OK;
}

int selfgpu_model2d_closure_state(selfgpu_model2d* m, double* nu, float* activation, float* indicatorActivation,
                                  int* counts, int resetCounts) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_closure_state: null handle");
  if (!m->avNu) return set_error(SELFGPU_ERR_STATE, "selfgpu_model2d_closure_state: no closure has been set");
  const size_t nEl = (size_t)m->nEl;
  cudaError_t e = cudaSuccess;
  if (nu) e = cudaMemcpyAsync(nu, m->avNu, nEl * sizeof(double), cudaMemcpyDeviceToDevice, m->stream);
  if (e == cudaSuccess && activation)
    e = cudaMemcpyAsync(activation, m->avAct, nEl * sizeof(float), cudaMemcpyDeviceToDevice, m->stream);
  if (e == cudaSuccess && indicatorActivation)
    e = cudaMemcpyAsync(indicatorActivation, m->avAct + nEl, nEl * sizeof(float), cudaMemcpyDeviceToDevice,
                        m->stream);
  if (e == cudaSuccess && counts) {
    e = cudaMemcpyAsync(counts, m->avFallbacks, 2 * sizeof(int), cudaMemcpyDeviceToHost, m->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  }
  if (e == cudaSuccess && resetCounts) e = cudaMemsetAsync(m->avFallbacks, 0, 2 * sizeof(int), m->stream);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_closure_state", e);
  return SELFGPU_OK;
}

int selfgpu_cig2d_closure_features(const double* q, int N, int nEl, const double* controlPoints,
                                   const double* qWeights, double s0, double kappa, float* activation,
                                   float* features, void* stream) {
  if (!q || N < 1 || N > SELFGPU_MAX_N || nEl < 1 || !controlPoints || !qWeights || !(kappa > 0.0))
    return set_error(SELFGPU_ERR_ARG, "selfgpu_cig2d_closure_features: bad arguments");
  if (features && N < 5) return set_error(SELFGPU_ERR_ARG, "selfgpu_cig2d_closure_features: features need N >= 5");
  AvArgs x{};
  x.s0 = s0;
  x.kappa = kappa;
  modal_matrix(N, controlPoints, qWeights, x.T);
  cudaError_t e = launch_closure_features(q, N + 1, nEl, x, activation, features, (cudaStream_t)stream);
  if (e != cudaSuccess) return fail_cuda("selfgpu_cig2d_closure_features", e);
  return SELFGPU_OK;
}

int selfgpu_model2d_set_halo(selfgpu_model2d* m, int nHalo) {
  if (!m || nHalo < 0) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_halo: bad arguments");
  if (m->avMode != AV_OFF)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_set_halo: the closure is single-rank");
  if (m->stream) cudaStreamSynchronize(m->stream);
  m->drop_graphs();
  m->nHalo = nHalo;
  cudaError_t e = m->alloc_caches();
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_set_halo", e);
  m->haveGeometry = false;  // sideInfo is validated against the new neighbour range
  m->valid = false;
  return SELFGPU_OK;
}

int selfgpu_model2d_prologue(selfgpu_model2d* m) {
  int rc = check_ready(m, "selfgpu_model2d_prologue");
  if (rc) return rc;
  cudaError_t e = m->prologue();
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_prologue", e);
  return SELFGPU_OK;
}

int selfgpu_model2d_stage(selfgpu_model2d* m, double dt, int stage) {
  int rc = check_ready(m, "selfgpu_model2d_stage");
  if (rc) return rc;
  if (stage < 0 || stage > 2) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_stage: stage must be 0, 1 or 2");
  if (!m->valid)
    return set_error(SELFGPU_ERR_STATE, "selfgpu_model2d_stage: the trace caches are stale (call "
                                        "selfgpu_model2d_prologue after setting the solution)");
  cudaError_t e = m->stage_once(dt, stage);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_stage", e);
  return SELFGPU_OK;
}

int selfgpu_model2d_caches(selfgpu_model2d* m, void** traces, int* traceBlockBytes, void** velocity,
                           int* velocityBlockBytes) {
  if (!m) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_caches: null handle");
  if (traces) *traces = m->tr[m->cur];
  if (traceBlockBytes) *traceBlockBytes = (int)m->trace_block_bytes();
  if (velocity) *velocity = (m->model == SELFGPU_MODEL_SW) ? m->vel[m->vcur] : nullptr;
  if (velocityBlockBytes) *velocityBlockBytes = (m->model == SELFGPU_MODEL_SW) ? (int)m->vel_block_bytes() : 0;
  return SELFGPU_OK;
}

int selfgpu_pack_blocks(const void* cache, const int* blocks, int n, int blockBytes, void* out, void* stream) {
  if (!cache || !blocks || n < 0 || blockBytes < 4 || blockBytes % 4 || !out)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_pack_blocks: bad arguments");
  if (n == 0) return SELFGPU_OK;
  const int words = blockBytes / 4;
  const long long total = (long long)n * words;
  k_move_blocks<<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
      (const uint32_t*)cache, blocks, n, words, (uint32_t*)out, 0);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda("selfgpu_pack_blocks", e);
  return SELFGPU_OK;
}

int selfgpu_unpack_blocks(const void* packed, const int* blocks, int n, int blockBytes, void* cache, void* stream) {
  if (!cache || !blocks || n < 0 || blockBytes < 4 || blockBytes % 4 || !packed)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_unpack_blocks: bad arguments");
  if (n == 0) return SELFGPU_OK;
  const int words = blockBytes / 4;
  const long long total = (long long)n * words;
  k_move_blocks<<<(int)std::min<long long>((total + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
      (const uint32_t*)packed, blocks, n, words, (uint32_t*)cache, 1);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda("selfgpu_unpack_blocks", e);
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

int selfgpu_model2d_entropy(selfgpu_model2d* m, double* entropy) {
  int rc = check_ready(m, "selfgpu_model2d_entropy");
  if (rc) return rc;
  if (!entropy) return set_error(SELFGPU_ERR_ARG, "selfgpu_model2d_entropy: null output");
  const double* aux = nullptr;
  if (m->model == SELFGPU_MODEL_LSW) aux = m->base.fld[0];
  else if (m->model == SELFGPU_MODEL_SW) aux = m->base.fld[2];
  if (!m->haveInterp) return set_error(SELFGPU_ERR_STATE, "selfgpu_model2d_entropy: no interpolant");
  cudaError_t e = cudaSuccess;
  if (!m->entropyBuf) e = cudaMalloc(&m->entropyBuf, ((size_t)m->nEl + 1) * sizeof(double));
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_entropy", e);
  QwArr w{};
  for (int k = 0; k < m->P; ++k) w.w[k] = m->base.qw[k];
  const int blocks = (m->nEl + 127) / 128 < 1184 ? (m->nEl + 127) / 128 : 1184;
  k_entropy_elements<<<blocks, 128, 0, m->stream>>>(m->model, m->base.q, m->base.J, aux, w, m->P, m->nEl, m->base.g,
                                                    m->base.gamma, m->entropyBuf);
  k_sum_block<<<1, 1024, 0, m->stream>>>(m->entropyBuf, m->nEl, m->entropyBuf + m->nEl);
  m->launches += 2;
  double h = 0.0;
  e = cudaMemcpyAsync(&h, m->entropyBuf + m->nEl, sizeof(double), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return fail_cuda("selfgpu_model2d_entropy", e);
  *entropy = h;
  return SELFGPU_OK;
}

// One block: every thread sums a strided subset of the elements, each element
// in the reference's node order, then a shared-memory tree (fixed order).
__global__ void __launch_bounds__(1024) k_integral_block(const double* __restrict__ f, int var, int nVar,
                                                         const double* __restrict__ J, QwArr qw, int P, int nEl,
                                                         double* out) {
  __shared__ double part[1024];
  const int PP = P * P;
  double s = 0.0;
  for (long long e = threadIdx.x; e < nEl; e += blockDim.x) {
    const double* fe = f + (size_t)PP * (var + (size_t)nVar * e);
    double se = 0.0;
    for (int j = 0; j < P; ++j)
      for (int i = 0; i < P; ++i) se = se + fe[i + P * j] * qw.w[i] * qw.w[j] * J[i + P * j + (size_t)PP * e];
    s += se;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = part[0];
}

int selfgpu_integral_mapped_scalar2d(const double* interior, int iVar, int nVar, const double* J,
                                     const double* qWeights, int N, int nEl, double* result, void* stream) {
  if (!interior || !J || !qWeights || !result || N < 1 || N > SELFGPU_MAX_N || nEl < 1 || nVar < 1 || iVar < 1 ||
      iVar > nVar)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_integral_mapped_scalar2d: bad arguments");
  QwArr w{};
  for (int k = 0; k <= N; ++k) w.w[k] = qWeights[k];
  double* d = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMallocAsync(&d, sizeof(double), st);
  if (e != cudaSuccess) return fail_cuda("selfgpu_integral_mapped_scalar2d", e);
  k_integral_block<<<1, 1024, 0, st>>>(interior, iVar - 1, nVar, J, w, N + 1, nEl, d);
  e = cudaGetLastError();
  double h = 0.0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h, d, sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail_cuda("selfgpu_integral_mapped_scalar2d", e);
  *result = h;
  return SELFGPU_OK;
}

long long selfgpu_model2d_launch_count(const selfgpu_model2d* m) { return m ? m->launches : 0; }

}  // extern "C"

// ----------------------------------------------------------------- ensembles
// Several handles advanced together: one RK step of all of them is ONE CUDA
// graph whose branches (one per handle, each on its own capture stream) hold
// that handle's stage launches, so the handles' kernels run concurrently and
// the whole ensemble costs one graph launch per step.  Captured per joint
// buffer parity of the handles (the parities flip every step, so two graphs
// serve a run) and re-captured when dt or any handle's launch state changes.
struct selfgpu_ensemble {
  std::vector<selfgpu_model2d*> h;
  cudaStream_t stream = nullptr;  // the stream the graph is launched on
  bool ownStream = false;
  std::vector<cudaStream_t> branch;  // capture streams, one per handle
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  struct Entry {
    std::vector<int> key;                  // (cur, vcur) of every handle at the step's start
    std::vector<unsigned long long> gen;   // handle generations at capture
    std::vector<long long> launches, tma;  // per handle and step
    double dt = NAN;
    cudaGraphExec_t g = nullptr;
  };
  std::vector<Entry> cache;

  std::vector<int> key() const {
    std::vector<int> k(h.size());
    for (size_t i = 0; i < h.size(); ++i) k[i] = h[i]->cur | (h[i]->vcur << 1);
    return k;
  }
  void drop() {
    for (auto& c : cache)
      if (c.g) cudaGraphExecDestroy(c.g);
    cache.clear();
  }
  Entry* find(double dt) {
    const std::vector<int> k = key();
    for (auto& c : cache) {
      if (c.key != k || !(c.dt == dt)) continue;
      bool fresh = true;
      for (size_t i = 0; i < h.size(); ++i) fresh = fresh && c.gen[i] == h[i]->gen;
      if (fresh) return &c;
    }
    return nullptr;
  }
  // capture one step of every handle from the current parities (restored afterwards)
  cudaError_t capture(double dt, Entry& out) {
    const size_t n = h.size();
    out.key = key();
    out.gen.resize(n);
    out.launches.assign(n, 0);
    out.tma.assign(n, 0);
    out.dt = dt;
    std::vector<int> c0(n), v0(n);
    std::vector<cudaStream_t> s0(n);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    e = cudaEventRecord(fork, stream);
    for (size_t i = 0; i < n && e == cudaSuccess; ++i) {
      selfgpu_model2d* m = h[i];
      c0[i] = m->cur;
      v0[i] = m->vcur;
      s0[i] = m->stream;
      out.gen[i] = m->gen;
      e = cudaStreamWaitEvent(branch[i], fork, 0);
      if (e != cudaSuccess) break;
      m->stream = branch[i];
      const long long l0 = m->launches, t0 = m->tmaLaunches;
      e = m->step(dt);
      out.launches[i] = m->launches - l0;
      out.tma[i] = m->tmaLaunches - t0;
      m->launches = l0;
      m->tmaLaunches = t0;
      m->stream = s0[i];
      m->cur = c0[i];
      m->vcur = v0[i];
      if (e == cudaSuccess) e = cudaEventRecord(join[i], branch[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, join[i], 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(stream, &graph);
    if (e == cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&out.g, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      cudaGetLastError();
      out.g = nullptr;
    }
    return e;
  }
};

extern "C" {

int selfgpu_ensemble_create(selfgpu_model2d* const* handles, int n, void* stream, selfgpu_ensemble** out) {
  if (!handles || n < 1 || !out) return set_error(SELFGPU_ERR_ARG, "selfgpu_ensemble_create: bad arguments");
  *out = nullptr;
  for (int i = 0; i < n; ++i) {
    if (!handles[i]) return set_error(SELFGPU_ERR_ARG, "selfgpu_ensemble_create: null handle");
    for (int k = 0; k < i; ++k)
      if (handles[k] == handles[i]) return set_error(SELFGPU_ERR_ARG, "selfgpu_ensemble_create: repeated handle");
  }
  auto* x = new selfgpu_ensemble();
  x->h.assign(handles, handles + n);
  cudaError_t e = cudaSuccess;
  if (stream) {
    x->stream = (cudaStream_t)stream;
  } else {
    e = cudaStreamCreateWithFlags(&x->stream, cudaStreamNonBlocking);
    x->ownStream = e == cudaSuccess;
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x->fork, cudaEventDisableTiming);
  x->branch.assign(n, nullptr);
  x->join.assign(n, nullptr);
  for (int i = 0; i < n && e == cudaSuccess; ++i) {
    e = cudaStreamCreateWithFlags(&x->branch[i], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&x->join[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    selfgpu_ensemble_destroy(x);
    return fail_cuda("selfgpu_ensemble_create", e);
  }
  *out = x;
  return SELFGPU_OK;
}

int selfgpu_ensemble_destroy(selfgpu_ensemble* x) {
  if (!x) return SELFGPU_OK;
  if (x->stream) cudaStreamSynchronize(x->stream);
  x->drop();
  for (auto s : x->branch)
    if (s) cudaStreamDestroy(s);
  for (auto ev : x->join)
    if (ev) cudaEventDestroy(ev);
  if (x->fork) cudaEventDestroy(x->fork);
  if (x->ownStream) cudaStreamDestroy(x->stream);
  delete x;
  return SELFGPU_OK;
}

int selfgpu_ensemble_rk3(selfgpu_ensemble* x, double dt, int nSteps) {
  if (!x || nSteps < 0) return set_error(SELFGPU_ERR_ARG, "selfgpu_ensemble_rk3: bad arguments");
  const size_t n = x->h.size();
  for (auto m : x->h) {
    int rc = check_ready(m, "selfgpu_ensemble_rk3");
    if (rc) return rc;
  }
  if (nSteps == 0) return SELFGPU_OK;
  cudaError_t e = cudaSuccess;
  // work already issued on the handles' streams (prologues included) comes first
  for (size_t i = 0; i < n && e == cudaSuccess; ++i) {
    selfgpu_model2d* m = x->h[i];
    if (!m->valid) e = m->prologue();
    if (e == cudaSuccess) e = cudaEventRecord(x->join[i], m->stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(x->stream, x->join[i], 0);
  }
  if (e != cudaSuccess) return fail_cuda("selfgpu_ensemble_rk3", e);
  for (int s = 0; s < nSteps; ++s) {
    selfgpu_ensemble::Entry* c = x->find(dt);
    if (!c) {
      if (x->cache.size() >= 4) x->drop();
      selfgpu_ensemble::Entry fresh;
      e = x->capture(dt, fresh);
      if (e != cudaSuccess) return fail_cuda("selfgpu_ensemble_rk3: capture", e);
      x->cache.push_back(std::move(fresh));
      c = &x->cache.back();
    }
    e = cudaGraphLaunch(c->g, x->stream);
    if (e != cudaSuccess) return fail_cuda("selfgpu_ensemble_rk3: graph launch", e);
    for (size_t i = 0; i < n; ++i) {
      selfgpu_model2d* m = x->h[i];
      m->launches += c->launches[i];
      m->tmaLaunches += c->tma[i];
      m->cur = 1 - m->cur;  // three swaps per step
      if (m->model == SELFGPU_MODEL_SW) m->vcur = 1 - m->vcur;
    }
  }
  // later work on the handles' streams waits for the steps
  e = cudaEventRecord(x->fork, x->stream);
  for (size_t i = 0; i < n && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(x->h[i]->stream, x->fork, 0);
  if (e != cudaSuccess) return fail_cuda("selfgpu_ensemble_rk3", e);
  return SELFGPU_OK;
}

}  // extern "C"
