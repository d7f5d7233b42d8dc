// A CompressibleIdealGas2D tendency entry point that allocates no memory.
//
// selfgpu_model2d_tendency keeps its face-trace cache in memory the engine
// allocates when the handle is created.  Some callers cannot allow any device
// allocation at the moment they need a tendency: a host code that hands the
// library all of its device memory up front and forbids the library from
// growing it, a caller running under a fixed memory cap (an MPS client
// limit, a pool reserved for one solver), or a call site deep inside a solver
// step that must not stall or fail on cudaMalloc.  For them this file keeps
// the scratch it needs -- the face-trace buffer written by one launch and read
// by the next -- in a fixed, file-scope device array of the library's device
// code.  The caller still passes every input and output buffer.
//
// Costs and limits of that choice:
//  * every GPU on which the entry point has been called holds
//    SELFGPU_NOALLOC_SCRATCH_BYTES (16 MiB) of device memory for this array
//    until the process exits;
//  * the array is shared by all calls on a device: two calls whose launches
//    overlap on the GPU (different streams, or different host threads) race
//    on it and produce wrong results -- serialise them;
//  * the array keeps the last call's contents.  Nothing in it needs to start
//    at zero: the first launch of each call writes every entry the second
//    launch reads;
//  * CUDA loads a module's device code lazily by default, so the array is
//    reserved on a device by the first call there (its address lookup), not
//    when the library is loaded: make one call on each device during set-up,
//    before any stream capture that is to contain later calls.  The first
//    call resolves the array's device address with cudaGetSymbolAddress
//    (with that device current); a failed lookup is not kept, the next call
//    tries again;
//  * the tendency has no gravity, drag or prescribed-boundary fields: sides
//    are periodic / interior (bcid 0) or NONORMALFLOW walls, and any other
//    physical side (PRESCRIBED, RADIATION, ...) is rejected, since its
//    exterior state would be zero (zero density) here.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "fused_stage.cuh"
#include "selfgpu_internal.h"

namespace selfgpu {
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SELFGPU_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

// Values per (element, side) block of the CompressibleIdealGas2D FP64 trace
// layout: 9 traced fields x P nodes, padded to 16 bytes.
int trace_block(int N) { return (9 * (N + 1) + 1) / 2 * 2; }
std::mutex g_scratch_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on `dev` (the current device).  Only a
// successful lookup is kept; after a failure (for instance a first call made
// during stream capture) the next call looks it up again.
cudaError_t scratch_address(int dev, void** out) {
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_ptr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      *out = nullptr;
      return e != cudaSuccess ? e : cudaErrorInvalidSymbol;
    }
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return cudaSuccess;
}

template <int P>
cudaError_t launch_pair(StageArgs a, cudaStream_t st) {
  constexpr int EPB = []() {
    int e = 128 / (P * P);
    if (e < 1) e = 1;
    while (e > 1 && (size_t)e * sizeof(Smem<P, PhysCIG, double>) > 44 * 1024) --e;
    return e;
  }();
  const int grid = (a.nEl + EPB - 1) / EPB;
  StageArgs t = a;
  t.mode = MODE_TRACES;
  t.trIn = nullptr;
  k_fused_stage<P, PhysCIG, double, EPB><<<grid, EPB * P * P, 0, st>>>(t);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  a.mode = MODE_TENDENCY;
  a.trIn = a.trOut;
  a.trOut = nullptr;
  k_fused_stage<P, PhysCIG, double, EPB><<<grid, EPB * P * P, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace
}  // namespace selfgpu

using namespace selfgpu;

extern "C" int selfgpu_cig2d_tendency_noalloc(const double* solution, double* dSdt, const double* dsdx,
                                              const double* J, const double* nHat, const double* nScale,
                                              const int* sideInfo_d, const int* sideInfo_h, const double* dgMatrix,
                                              const double* bMatrix, const double* qWeights,
                                              double expansionFactor, int N, int nEl, void* stream) {
  if (!solution || !dSdt || !dsdx || !J || !nHat || !nScale || !sideInfo_d || !sideInfo_h || !dgMatrix ||
      !bMatrix || !qWeights)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_cig2d_tendency_noalloc: null argument");
  if (N < 1 || N > SELFGPU_MAX_N || nEl < 1)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_cig2d_tendency_noalloc: N must be in 1..7 and nEl >= 1");
  const int P = N + 1;
  const long long need = 4LL * nEl * trace_block(N) * (long long)sizeof(double);
  if (need > SELFGPU_NOALLOC_SCRATCH_BYTES)
    return set_error(SELFGPU_ERR_ARG,
                     "selfgpu_cig2d_tendency_noalloc: " + std::to_string(nEl) + " elements at N = " +
                         std::to_string(N) + " need " + std::to_string(need) + " bytes of scratch; the fixed limit is " +
                         std::to_string((long long)SELFGPU_NOALLOC_SCRATCH_BYTES) + " bytes (" +
                         std::to_string(SELFGPU_NOALLOC_SCRATCH_BYTES / (4LL * trace_block(N) * 8)) +
                         " elements at this degree)");
  if (((uintptr_t)dsdx % 16) || ((uintptr_t)nHat % 16))
    return set_error(SELFGPU_ERR_ARG, "selfgpu_cig2d_tendency_noalloc: dsdx and nHat must be 16-byte aligned");
  int rc = validate_side_info(sideInfo_h, nEl, nEl);
  if (rc != SELFGPU_OK) return rc;
  // physical sides (no neighbour element) must be NONORMALFLOW walls: there
  // are no prescribed traces here, and any other boundary condition would see
  // a zero exterior state
  for (long long k = 0; k < 4LL * nEl; ++k) {
    const int* si = sideInfo_h + 5 * k;
    if (si[2] == 0 && si[4] != 0 && si[4] != SELFGPU_BC_NONORMALFLOW)
      return set_error(SELFGPU_ERR_ARG, "selfgpu_cig2d_tendency_noalloc: side " + std::to_string(k % 4 + 1) +
                                            " of element " + std::to_string(k / 4 + 1) + " has boundary condition " +
                                            std::to_string(si[4]) +
                                            "; only periodic/interior sides and NONORMALFLOW walls are supported");
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return set_error(SELFGPU_ERR_CUDA, "selfgpu_cig2d_tendency_noalloc: no usable current device");
  void* scratch = nullptr;
  e = scratch_address(dev, &scratch);
  if (e != cudaSuccess || scratch == nullptr)
    return set_error(SELFGPU_ERR_CUDA, std::string("selfgpu_cig2d_tendency_noalloc: cudaGetSymbolAddress: ") +
                                           cudaGetErrorString(e));
  StageArgs a{};
  a.nEl = nEl;
  a.dsdx = dsdx;
  a.J = J;
  a.nHat = nHat;
  a.nScale = nScale;
  a.sideInfo = sideInfo_d;
  a.q = const_cast<double*>(solution);  // read only in both launches
  a.dSdt = dSdt;
  a.trOut = scratch;
  a.gamma = expansionFactor;
  a.g = 1.0;     // no gravity field is bound, so g never enters the tendency
  a.Rgas = 1.0;  // the gas constant only enters the (unused) temperature diagnostic
  for (int k = 0; k < P * P; ++k) a.dgM[k] = dgMatrix[k];
  for (int k = 0; k < 2 * P; ++k) a.bM[k] = bMatrix[k];
  for (int k = 0; k < P; ++k) a.qw[k] = qWeights[k];
  cudaStream_t st = (cudaStream_t)stream;
  switch (P) {
    case 2: e = launch_pair<2>(a, st); break;
    case 3: e = launch_pair<3>(a, st); break;
    case 4: e = launch_pair<4>(a, st); break;
    case 5: e = launch_pair<5>(a, st); break;
    case 6: e = launch_pair<6>(a, st); break;
    case 7: e = launch_pair<7>(a, st); break;
    default: e = launch_pair<8>(a, st); break;
  }
  if (e != cudaSuccess)
    return set_error(SELFGPU_ERR_CUDA, std::string("selfgpu_cig2d_tendency_noalloc: ") + cudaGetErrorString(e));
  return SELFGPU_OK;
}
