// Host-side launch of the fused stage kernels for one bulk type R.  Included
// by stage_fp64.cu (built with -fmad=false so that every FP64 operation rounds
// exactly as the reference's CPU path does), stage_fp64_prod.cu (the
// production FP64 form) and stage_fp32.cu.  The launchers sit in the build's
// form namespace (physics.cuh), so each build launches its own kernels.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "fused_stage.cuh"
#include "fused_stage_tma.cuh"
#include "selfgpu_internal.h"

namespace selfgpu {
inline namespace SELFGPU_FORM_NS {

template <int P, class Phys, typename R>
constexpr int elems_per_block() {
  int e = 128 / (P * P);
  if (e < 1) e = 1;
  while (e > 1 && (size_t)e * sizeof(Smem<P, Phys, R>) > 44 * 1024) --e;
  return e;
}

inline bool aligned16(const void* p) { return ((uintptr_t)p % 16) == 0; }

template <int P, class Phys, typename R>
cudaError_t launch_one(const StageArgs& a, const StageLaunch& L, cudaStream_t st, int* usedTma) {
  *usedTma = 0;
  if constexpr (P % 2 == 0) {
    bool ok = L.allowTma && a.mode != MODE_TRACES && a.geo != nullptr && aligned16(a.geo) && aligned16(a.q) &&
              aligned16(sizeof(R) == 4 ? (const void*)a.Gf : (const void*)a.G) && aligned16(a.trIn) &&
              (a.velIn == nullptr || aligned16(a.velIn));
    for (int k = 0; k < 5; ++k) ok = ok && (a.fld[k] == nullptr || aligned16(a.fld[k]));
    TmaPlan pl{};
    if (ok && make_tma_plan<P, Phys, R>(a, L.smemOptin, pl, L.maxGroups)) {
      // the shared-memory opt-in is per device: one bit per device that has it
      static std::atomic<unsigned long long> attrSet{0};  // one instantiation per (P, Phys, R)
      int dev = 0;
      cudaError_t e = cudaGetDevice(&dev);
      if (e != cudaSuccess) return e;
      const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
      if (!(attrSet.load() & bit)) {
        e = cudaFuncSetAttribute(k_fused_stage_tma<P, Phys, R>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 L.smemOptin);
        if (e != cudaSuccess) return e;
        attrSet.fetch_or(bit);
      }
      using T = TmaTraits<P, Phys, R>;
      const int tiles = (a.nEl + T::EPG - 1) / T::EPG;  // work items of EPG consecutive elements
      const int grid = tiles < L.numSMs ? tiles : L.numSMs;
      // Programmatic dependent launch: the launch and the kernel's prologue
      // overlap the end of the previous kernel on the stream; the kernel waits
      // for that kernel's completion (griddepcontrol.wait) before it touches
      // any data the previous kernel may write or read.
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(grid);
      cfg.blockDim = dim3(pl.groups * T::TPE);
      cfg.dynamicSmemBytes = pl.smemBytes;
      cfg.stream = st;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      *usedTma = 1;
      const TmaSteps none{};
      return cudaLaunchKernelEx(&cfg, k_fused_stage_tma<P, Phys, R>, a, pl, none);
    }
  }
  constexpr int EPB = elems_per_block<P, Phys, R>();
  const int grid = (a.nEl + EPB - 1) / EPB;
  k_fused_stage<P, Phys, R, EPB><<<grid, EPB * P * P, 0, st>>>(a);
  return cudaGetLastError();
}

// ms.nStages RK stages in one cooperative launch of the persistent kernel
// (k_fused_stage_tma<..., true>).  cudaErrorNotSupported where it does not
// apply (P != 8, unaligned buffers, a mesh that gives some group fewer than
// three or more than 24 tiles per stage), cudaErrorCooperativeLaunchTooLarge when the CTAs
// cannot all be resident; the caller then falls back to stage launches.
template <int P, class Phys, typename R>
cudaError_t launch_stages_tma_one(const StageArgs& a, const StageLaunch& L, TmaSteps ms, cudaStream_t st) {
  if constexpr (TmaTraits<P, Phys, R>::EPG != 1) {
    return cudaErrorNotSupported;
  } else {
    bool ok = L.allowTma && a.geo != nullptr && aligned16(a.geo) && aligned16(a.q) &&
              aligned16(sizeof(R) == 4 ? (const void*)a.Gf : (const void*)a.G) &&
              aligned16(ms.tr[0]) && aligned16(ms.tr[1]) && (ms.vel[0] == nullptr || aligned16(ms.vel[0])) &&
              (ms.vel[1] == nullptr || aligned16(ms.vel[1])) && a.av == 0 && a.debugStarve != 1;
    for (int k = 0; k < 5; ++k) ok = ok && (a.fld[k] == nullptr || aligned16(a.fld[k]));
    TmaPlan pl{};
    if (!ok || !make_tma_plan<P, Phys, R>(a, L.smemOptin, pl, L.maxGroups)) return cudaErrorNotSupported;
    using T = TmaTraits<P, Phys, R>;
    const long long tiles = ((long long)a.nEl + T::EPG - 1) / T::EPG;
    const int grid = tiles < L.numSMs ? (int)tiles : L.numSMs;
    // every group of every CTA needs three tiles per stage (the copies of the
    // next stage's first two tiles read what the group's earlier tiles wrote);
    // beyond 24 per group the per-launch costs this launch saves are small
    // against the stage (measured: 1.04x at 11 tiles per group, C2, and
    // within +-2 % at 44) and stage launches are kept
    if (grid < 1 || tiles / grid < 3LL * pl.groups || tiles > 24LL * pl.groups * grid) return cudaErrorNotSupported;
    static std::atomic<unsigned long long> attrSet{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (!(attrSet.load() & bit)) {
      e = cudaFuncSetAttribute(k_fused_stage_tma<P, Phys, R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               L.smemOptin);
      if (e != cudaSuccess) return e;
      attrSet.fetch_or(bit);
    }
    ms.nGroups = grid * pl.groups;
    StageArgs aa = a;
    aa.mode = MODE_RK;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(pl.groups * T::TPE);
    cfg.dynamicSmemBytes = pl.smemBytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;  // all CTAs resident: the stage-end waits need it
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_fused_stage_tma<P, Phys, R, true>, aa, pl, ms);
  }
}

// P = 8 only: its tiles have one face warp (the stage-end wait is that
// warp's); at P = 4 and 6 the launch measured slower than stage launches.
template <class Phys, typename R>
cudaError_t launch_stages_tma_P(int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                cudaStream_t st) {
  return P == 8 ? launch_stages_tma_one<8, Phys, R>(a, L, ms, st) : cudaErrorNotSupported;
}

template <typename R>
cudaError_t launch_stages_tma_impl(int model, int P, const StageArgs& a, const StageLaunch& L, const TmaSteps& ms,
                                   cudaStream_t st) {
  switch (model) {
    case SELFGPU_MODEL_LSW: return launch_stages_tma_P<PhysLSW, R>(P, a, L, ms, st);
    case SELFGPU_MODEL_SW: return launch_stages_tma_P<PhysSW, R>(P, a, L, ms, st);
    case SELFGPU_MODEL_CIG: return launch_stages_tma_P<PhysCIG, R>(P, a, L, ms, st);
    default: return cudaErrorInvalidValue;
  }
}

template <class Phys, typename R>
cudaError_t launch_P(int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st, int* usedTma) {
  switch (P) {
    case 2: return launch_one<2, Phys, R>(a, L, st, usedTma);
    case 3: return launch_one<3, Phys, R>(a, L, st, usedTma);
    case 4: return launch_one<4, Phys, R>(a, L, st, usedTma);
    case 5: return launch_one<5, Phys, R>(a, L, st, usedTma);
    case 6: return launch_one<6, Phys, R>(a, L, st, usedTma);
    case 7: return launch_one<7, Phys, R>(a, L, st, usedTma);
    case 8: return launch_one<8, Phys, R>(a, L, st, usedTma);
    default: return cudaErrorInvalidValue;
  }
}

// One cooperative launch of k_fused_steps; cudaErrorCooperativeLaunchTooLarge
// when the element groups do not fit one wave of resident CTAs.
template <int P, class Phys, typename R>
cudaError_t launch_steps_one(const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st) {
  constexpr int EPB = elems_per_block<P, Phys, R>();
  const int grid = (a.nEl + EPB - 1) / EPB;
  int perSM = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k_fused_steps<P, Phys, R, EPB>, EPB * P * P, 0);
  if (e != cudaSuccess) return e;
  if ((long long)perSM * numSMs < grid) return cudaErrorCooperativeLaunchTooLarge;
  StageArgs aa = a;
  StepsArgs ss = sa;
  void* args[] = {&aa, &ss};
  return cudaLaunchCooperativeKernel((const void*)k_fused_steps<P, Phys, R, EPB>, dim3(grid), dim3(EPB * P * P),
                                     args, 0, st);
}

template <class Phys, typename R>
cudaError_t launch_steps_P(int P, const StageArgs& a, const StepsArgs& sa, int numSMs, cudaStream_t st) {
  switch (P) {
    case 2: return launch_steps_one<2, Phys, R>(a, sa, numSMs, st);
    case 3: return launch_steps_one<3, Phys, R>(a, sa, numSMs, st);
    case 4: return launch_steps_one<4, Phys, R>(a, sa, numSMs, st);
    case 5: return launch_steps_one<5, Phys, R>(a, sa, numSMs, st);
    case 6: return launch_steps_one<6, Phys, R>(a, sa, numSMs, st);
    case 7: return launch_steps_one<7, Phys, R>(a, sa, numSMs, st);
    case 8: return launch_steps_one<8, Phys, R>(a, sa, numSMs, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
cudaError_t launch_steps_impl(int model, int P, const StageArgs& a, const StepsArgs& sa, int numSMs,
                              cudaStream_t st) {
  switch (model) {
    case SELFGPU_MODEL_LSW: return launch_steps_P<PhysLSW, R>(P, a, sa, numSMs, st);
    case SELFGPU_MODEL_SW: return launch_steps_P<PhysSW, R>(P, a, sa, numSMs, st);
    case SELFGPU_MODEL_CIG: return launch_steps_P<PhysCIG, R>(P, a, sa, numSMs, st);
    default: return cudaErrorInvalidValue;
  }
}

template <typename R>
cudaError_t launch_stage_impl(int model, int P, const StageArgs& a, const StageLaunch& L, cudaStream_t st,
                              int* usedTma) {
  switch (model) {
    case SELFGPU_MODEL_LSW: return launch_P<PhysLSW, R>(P, a, L, st, usedTma);
    case SELFGPU_MODEL_SW: return launch_P<PhysSW, R>(P, a, L, st, usedTma);
    case SELFGPU_MODEL_CIG: return launch_P<PhysCIG, R>(P, a, L, st, usedTma);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace SELFGPU_FORM_NS
}  // namespace selfgpu
