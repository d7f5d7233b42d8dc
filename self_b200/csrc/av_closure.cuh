// Artificial-viscosity closure of the CompressibleIdealGas2D tendency.
//
// Not a reference routine: the shock closure built from the reference's own
// operators -- BassiRebaySides + GradientBR (src/SELF_MappedData.f90:919-1078),
// VectorBoundaryInterp (src/SELF_Lagrange.f90:2284-2316), SideExchange of a
// vector (src/SELF_MappedData.f90:1870-1958) and the Advection2D diffusive flux
// templates (src/models/hip/SELF_Advection2D.cpp:66-95, :140-175) -- with one
// viscosity per element instead of one diffusivity.
//
// With the closure on, each RK stage runs, before the stage kernel:
//   k_av_nu     (the first stage of an RK step, and a tendency evaluation;
//               the step's other two stages keep its viscosity and list) the
//               element viscosity nu (modal-decay indicator of the density,
//               or the closure MLP with the indicator as fallback and screen),
//               and the list of elements with nu > 0: one lane per element for
//               the indicator, warp-wide for the few elements that need the
//               MLP or the wave speed;
//   k_av_grad   the listed elements only: the BR1 gradient of the four
//               conservative variables from the averaged traces of the stage's
//               trace cache, the contravariant viscous volume flux
//               -(dsdx^T nu grad q) and the face traces of nu grad q;
//   the stage   kernel adds the viscous volume flux to its contravariant flux
//               and, on exchanged sides, -1/2 (nu grad q_in + nu grad q_ex) . n
//               nScale to its face flux, the exterior value coming from the
//               neighbour's traces; physical sides carry no viscous flux.
// Only elements with nu > 0 form the gradient and write viscous terms; the
// stage kernel reads them only where nu > 0 (the rest add exact zeros).
//
// Modal decay indicator (Persson & Peraire, AIAA 2006-112): c_kl are the
// orthonormal Legendre modes of the density, S = sum_{max(k,l)=N} c^2 /
// sum c^2, s = log10 S, activation a = 0 below s0 - kappa, 1 above s0 + kappa,
// (1 + sin(pi (s - s0) / (2 kappa))) / 2 between; nu = a c_av h / N lambda with
// lambda = max over nodes of |u| + c and h = sqrt(element area).
//
// Closure MLP: 36 features (per variable, density then total energy, the
// energy fractions of the six highest shells max(k,l), xi-degrees and
// eta-degrees, log-scaled) -> 32 -> 32 -> 1, ReLU, bfloat16 weights, float32
// accumulation, output clamp(z, 0, 1) replaces a.
#pragma once

#include <cuda_bf16.h>

#include <atomic>

#include "fused_stage.cuh"

namespace selfgpu {

constexpr int kMlpIn = 36, kMlpHidden = 32;
constexpr int kMlpWeights = kMlpHidden * kMlpIn + kMlpHidden * kMlpHidden + kMlpHidden;  // bf16 values
constexpr int kMlpFloats = kMlpHidden + kMlpHidden + 1 + 2 * kMlpIn;                    // b1 b2 b3 fmin fmax
constexpr double kAvPi = 3.141592653589793;                                             // 4 atan(1)
constexpr float kMlpRangeMargin = 0.05f;
// Screening: an element whose modal decay lies more than kMlpGate decades
// below the start of the activation ramp (s < s0 - kappa - kMlpGate) is smooth
// by a wide margin and gets a = 0 without evaluating the MLP.
constexpr double kMlpGate = 1.0;

enum AvMode { AV_OFF = 0, AV_INDICATOR = 1, AV_MLP = 2 };

struct AvArgs {
  int nEl;
  int mode;  // AV_INDICATOR or AV_MLP
  const double* q;
  const double* dsdx;
  const double* J;
  const double* nHat;
  const double* nScale;
  const int* sideInfo;
  const void* trIn;     // trace cache of this stage (bulk type); conservative traces are fields 0..3
  const double* presc;  // prescribed solution boundary (P,4,4,nEl) or null
  const double* hEl;    // element size sqrt(area), (nEl)
  double gamma, avC, s0, kappa;
  double* nu;          // element viscosity (nEl)
  float* act;          // activation applied (nEl)
  float* actInd;       // indicator activation (nEl), written in AV_MLP mode
  int* fallbacks;      // AV_MLP counters: [0] features outside the training range, [1] MLP evaluations
  int* activeCount;    // elements with nu > 0 in this stage (reset before the viscosity kernel)
  int* activeList;     // their ids (nEl capacity)
  void* visc;          // contravariant viscous volume flux (P*P, 2, 4, nEl), bulk type
  void* vtr;           // per (element, side): nu grad q traces at [i + P (d + 2 v)], bulk type
  const __nv_bfloat16* mlpW;  // W1 (32 x 36, row-major), W2 (32 x 32), w3 (32)
  const float* mlpB;          // b1 (32), b2 (32), b3, fmin (36), fmax (36)
  double T[kMaxP * kMaxP];    // modal matrix T(k,i) = w_i Lt_k(x_i) at [k + P i]
  double dgM[kMaxP * kMaxP];
  double bM[2 * kMaxP];
  double qw[kMaxP];
};

template <typename R>
__device__ __forceinline__ R av_log10(R x) {
  if constexpr (sizeof(R) == 8) return log10(x);
  else return log10f(x);
}
template <typename R>
__device__ __forceinline__ R av_sin(R x) {
  if constexpr (sizeof(R) == 8) return sin(x);
  else return sinf(x);
}
template <typename R>
__device__ __forceinline__ R av_sqrt(R x) {
  if constexpr (sizeof(R) == 8) return sqrt(x);
  else return sqrtf(x);
}

// Modal decay activation from one variable's modes c[k + P l] (one thread).
template <int P, typename R>
__device__ R modal_activation(const R* c, double s0, double kappa) {
  constexpr int N = P - 1;
  R top = (R)0, total = (R)0;
  for (int l = 0; l < P; ++l)
    for (int k = 0; k < P; ++k) {
      const R e = c[k + P * l] * c[k + P * l];
      total = total + e;
      if (k == N || l == N) top = top + e;
    }
  if (!(top > (R)0) || !(total > (R)0)) return (R)0;
  const R sv = av_log10<R>(top / total);
  if (sv < (R)s0 - (R)kappa) return (R)0;
  if (sv > (R)s0 + (R)kappa) return (R)1;
  return (R)0.5 * ((R)1 + av_sin<R>((R)kAvPi * (sv - (R)s0) / ((R)2 * (R)kappa)));
}

// The 18 features of one variable's modes (one thread); requires P >= 6.
template <int P, typename R>
__device__ void modal_features(const R* c, float* f) {
  constexpr int N = P - 1;
  R total = (R)0, sh[P], ex[P], ey[P];
#pragma unroll
  for (int k = 0; k < P; ++k) sh[k] = ex[k] = ey[k] = (R)0;
  for (int l = 0; l < P; ++l)
#pragma unroll
    for (int k = 0; k < P; ++k) {
      const R e = c[k + P * l] * c[k + P * l];
      total = total + e;
      const int m = k > l ? k : l;
      sh[m] = sh[m] + e;
      ex[k] = ex[k] + e;
      ey[l] = ey[l] + e;
    }
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const int m = N - 5 + r;
    const R fr[3] = {sh[m], ex[m], ey[m]};
#pragma unroll
    for (int g = 0; g < 3; ++g) {
      R q = total > (R)0 ? fr[g] / total : (R)0;
      if (q < (R)1e-16) q = (R)1e-16;
      f[r + 6 * g] = (float)((av_log10<R>(q) + (R)8) / (R)8);
    }
  }
}

// ------------------------------------------------------ viscosity kernel
// One lane per element: density modes, activation and screening; then, warp
// wide (warp-level synchronisation only) and only for the warp's elements
// that need them, the MLP where the indicator does not screen the element
// out, and the wave speed where the activation is not zero; the viscosity and
// an entry in the list of active elements.
template <int P, typename R>
struct NuWarpSmem {
  static constexpr int PP = P * P;
  R q[2][PP];  // density, total energy
  R tt[PP];
  R c[2][PP];  // modal energies c^2
  R part[3][P];
  R act[32], lam[32];  // per lane's element
  float feat[kMlpIn];
  float h1[kMlpHidden];
};

// Orthonormal modal energies of one P x P field of this warp's element:
// c(k,l) = sum_j T(l,j) sum_i T(k,i) q(i,j), then c^2 in place.
template <int P, typename R>
__device__ __forceinline__ void warp_modal_energy(const R* sT, const R* q, R* tt, R* c, int lane) {
  constexpr int PP = P * P;
  for (int o = lane; o < PP; o += 32) {
    const int k = o % P, jj = o / P;
    R acc = (R)0;
#pragma unroll
    for (int m = 0; m < P; ++m) acc = acc + sT[k + P * m] * q[m + P * jj];
    tt[k + P * jj] = acc;
  }
  __syncwarp();
  for (int o = lane; o < PP; o += 32) {
    const int k = o % P, l = o / P;
    R acc = (R)0;
#pragma unroll
    for (int m = 0; m < P; ++m) acc = acc + sT[l + P * m] * tt[k + P * m];
    c[k + P * l] = acc * acc;
  }
  __syncwarp();
}

constexpr int kNuWarps = 4;

// The closure MLP's activation for element e (warp-wide): the density and
// total-energy modes, the 36 features, the two hidden layers and the clamped
// output; the indicator activation actInd stays when a feature lies outside
// the training range (counted).  Lane 0's result is returned on every lane.
template <int P, typename R>
__device__ R warp_mlp_act(const AvArgs& a, const R* sT, NuWarpSmem<P, R>& s, const float* sW1, const float* sW2,
                          const float* sw3, const float* sB, long long e, int lane, R actInd) {
  constexpr int PP = P * P, N = P - 1;
  R act = actInd;
  for (int k = lane; k < PP; k += 32) {
    s.q[0][k] = (R)a.q[k + (long long)PP * (2 + 4 * e)];
    s.q[1][k] = (R)a.q[k + (long long)PP * (3 + 4 * e)];
  }
  __syncwarp();
  warp_modal_energy<P, R>(sT, s.q[0], s.tt, s.c[0], lane);
  warp_modal_energy<P, R>(sT, s.q[1], s.tt, s.c[1], lane);
  if (lane < P) {  // fixed-order sums per eta-degree l, then over l
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      R tot = (R)0;
#pragma unroll
      for (int k = 0; k < P; ++k) tot = tot + s.c[r][k + P * lane];
      s.part[r][lane] = tot;
    }
  }
  __syncwarp();
  if (lane < 2) {
    R total = (R)0;
#pragma unroll
    for (int l = 0; l < P; ++l) total = total + s.part[lane][l];
    s.part[2][lane] = total;
  }
  __syncwarp();
  for (int f = lane; f < kMlpIn; f += 32) {
    const int r = f / 18, grp = (f % 18) / 6, m = N - 5 + f % 6;
    const R* e2 = s.c[r];
    R sum = (R)0;
    if (grp == 0) {
      for (int l = 0; l < m; ++l) sum = sum + e2[m + P * l];
      for (int k = 0; k <= m; ++k) sum = sum + e2[k + P * m];
    } else if (grp == 1) {
      for (int l = 0; l < P; ++l) sum = sum + e2[m + P * l];
    } else {
      for (int k = 0; k < P; ++k) sum = sum + e2[k + P * m];
    }
    const R total = s.part[2][r];
    R qf = total > (R)0 ? sum / total : (R)0;
    if (qf < (R)1e-16) qf = (R)1e-16;
    s.feat[f] = (float)((av_log10<R>(qf) + (R)8) / (R)8);
  }
  __syncwarp();
  {
    float acc = 0.f;  // lane = hidden unit
#pragma unroll 4
    for (int k = 0; k < kMlpIn; ++k) acc = fmaf(sW1[lane * kMlpIn + k], s.feat[k], acc);
    acc = acc + sB[lane];
    s.h1[lane] = acc > 0.f ? acc : 0.f;
  }
  __syncwarp();
  float h2;
  {
    float acc = 0.f;
#pragma unroll 4
    for (int k = 0; k < kMlpHidden; ++k) acc = fmaf(sW2[lane * kMlpHidden + k], s.h1[k], acc);
    acc = acc + sB[kMlpHidden + lane];
    h2 = acc > 0.f ? acc : 0.f;
  }
  __syncwarp();
  s.h1[lane] = h2;  // the second hidden layer reuses the first's array
  __syncwarp();
  if (lane == 0) {
    if (a.fallbacks) atomicAdd(a.fallbacks + 1, 1);
    bool inRange = true;
    const float* fmin = sB + 2 * kMlpHidden + 1;
    const float* fmax = fmin + kMlpIn;
    for (int k = 0; k < kMlpIn; ++k)
      inRange = inRange && s.feat[k] >= fmin[k] - kMlpRangeMargin && s.feat[k] <= fmax[k] + kMlpRangeMargin;
    if (inRange) {
      float z = 0.f;
      for (int k = 0; k < kMlpHidden; ++k) z = fmaf(sw3[k], s.h1[k], z);
      z = z + sB[2 * kMlpHidden];
      act = (R)(z < 0.f ? 0.f : (z > 1.f ? 1.f : z));
    } else if (a.fallbacks) {
      atomicAdd(a.fallbacks, 1);
    }
  }
  act = __shfl_sync(0xffffffffu, act, 0);
  __syncwarp();
  return act;
}

// Wave speed |u| + c of element e, max over its nodes (warp-wide;
// src/models/SELF_CompressibleIdealGas2D.f90:1090-1110).
template <int P, typename R>
__device__ R warp_wave_speed(const AvArgs& a, long long e, int lane) {
  constexpr int PP = P * P;
  const R gam = (R)a.gamma;
  R lam = (R)0;
  for (int k = lane; k < PP; k += 32) {
    const long long b = k + (long long)PP * 4 * e;
    const R ru = (R)a.q[b], rv = (R)a.q[b + PP], rho = (R)a.q[b + 2 * PP], rE = (R)a.q[b + 3 * PP];
    const R u = ru / rho, v = rv / rho;
    const R ke = (R)0.5 * (ru * u + rv * v);
    const R p = (gam - (R)1) * (rE - ke);
    const R c = av_sqrt<R>(gam * p / rho);
    const R wv = av_sqrt<R>(u * u + v * v) + c;
    if (wv > lam) lam = wv;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const R other = __shfl_xor_sync(0xffffffffu, lam, o);
    if (other > lam) lam = other;
  }
  return lam;
}

// Indicator activation from the totals of all modal energies and of the top
// shell, and whether the MLP must be evaluated (not screened out).
template <typename R>
__device__ __forceinline__ void indicator_act(const AvArgs& a, R total, R top, bool mlp, R& actInd, int& need) {
  actInd = (R)0;
  need = 0;
  if (top > (R)0 && total > (R)0) {
    const R sv = av_log10<R>(top / total);
    if (sv > (R)a.s0 + (R)a.kappa) actInd = (R)1;
    else if (!(sv < (R)a.s0 - (R)a.kappa))
      actInd = (R)0.5 * ((R)1 + av_sin<R>((R)kAvPi * (sv - (R)a.s0) / ((R)2 * (R)a.kappa)));
    need = mlp && !(sv < (R)(a.s0 - a.kappa - kMlpGate));
  }
}

template <int P, typename R>
__global__ void __launch_bounds__(32 * kNuWarps) k_av_nu(const AvArgs a) {
  constexpr int PP = P * P, N = P - 1;
  __shared__ NuWarpSmem<P, R> ws[kNuWarps];
  __shared__ R sT[PP];
  __shared__ float sW1[kMlpHidden * kMlpIn], sW2[kMlpHidden * kMlpHidden], sw3[kMlpHidden], sB[kMlpFloats];
  const bool mlp = (a.mode == AV_MLP) && (P >= 6);
  for (int k = threadIdx.x; k < PP; k += blockDim.x) sT[k] = (R)a.T[k];
  if (mlp) {
    for (int k = threadIdx.x; k < kMlpHidden * kMlpIn; k += blockDim.x) sW1[k] = __bfloat162float(a.mlpW[k]);
    for (int k = threadIdx.x; k < kMlpHidden * kMlpHidden; k += blockDim.x)
      sW2[k] = __bfloat162float(a.mlpW[kMlpHidden * kMlpIn + k]);
    for (int k = threadIdx.x; k < kMlpHidden; k += blockDim.x)
      sw3[k] = __bfloat162float(a.mlpW[kMlpHidden * kMlpIn + kMlpHidden * kMlpHidden + k]);
    for (int k = threadIdx.x; k < kMlpFloats; k += blockDim.x) sB[k] = a.mlpB[k];
  }
  __syncthreads();
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  NuWarpSmem<P, R>& s = ws[w];
  {
    // One lane per element for the indicator (the warp's 32 elements are
    // spread over the mesh, so that the few that need the MLP or the wave
    // speed, done warp-wide, are spread over the warps too).  FP64 at P = 8
    // holds 64 densities per lane and spills a little; still measured 7 %
    // faster per C5 step than one warp per element.
    const long long nW = (long long)gridDim.x * kNuWarps;
    for (long long base = (long long)blockIdx.x * kNuWarps + w; base < a.nEl; base += 32 * nW) {
      const long long e = base + (long long)lane * nW;
      R actInd = (R)0;
      int need = 0;
      if (e < a.nEl) {
        // density modes: the operations and summation orders of warp_modal_energy
        // and of the per-eta-degree sums
        R q[PP];
        const double2* qg = reinterpret_cast<const double2*>(a.q + (long long)PP * (2 + 4 * e));
#pragma unroll
        for (int k = 0; k < PP / 2; ++k) {
          const double2 x = qg[k];
          q[2 * k] = (R)x.x;
          q[2 * k + 1] = (R)x.y;
        }
        if constexpr (PP % 2) q[PP - 1] = (R)a.q[(long long)PP * (2 + 4 * e) + PP - 1];
        R tot[P], top[P];
#pragma unroll
        for (int l = 0; l < P; ++l) tot[l] = top[l] = (R)0;
#pragma unroll
        for (int k = 0; k < P; ++k) {
          R tt[P];
#pragma unroll
          for (int jj = 0; jj < P; ++jj) {
            R acc = (R)0;
#pragma unroll
            for (int m = 0; m < P; ++m) acc = acc + sT[k + P * m] * q[m + P * jj];
            tt[jj] = acc;
          }
#pragma unroll
          for (int l = 0; l < P; ++l) {
            R acc = (R)0;
#pragma unroll
            for (int m = 0; m < P; ++m) acc = acc + sT[l + P * m] * tt[m];
            const R c = acc * acc;
            tot[l] = tot[l] + c;
            if (k == N) top[l] = c;
          }
        }
        top[N] = tot[N];
        R total = (R)0, topS = (R)0;
#pragma unroll
        for (int l = 0; l < P; ++l) {
          total = total + tot[l];
          topS = topS + top[l];
        }
        indicator_act<R>(a, total, topS, mlp, actInd, need);
      }
      s.act[lane] = actInd;
      const unsigned needMask = __ballot_sync(0xffffffffu, need);
      __syncwarp();
      for (unsigned mk = needMask; mk; mk &= mk - 1) {
        const int b = __ffs(mk) - 1;
        const R act = warp_mlp_act<P, R>(a, sT, s, sW1, sW2, sw3, sB, base + (long long)b * nW, lane,
                                         __shfl_sync(0xffffffffu, actInd, b));
        if (lane == 0) s.act[b] = act;
        __syncwarp();
      }
      const R act = s.act[lane];
      const unsigned actMask = __ballot_sync(0xffffffffu, e < a.nEl && act != (R)0);
      for (unsigned mk = actMask; mk; mk &= mk - 1) {
        const int b = __ffs(mk) - 1;
        const R lam = warp_wave_speed<P, R>(a, base + (long long)b * nW, lane);
        if (lane == 0) s.lam[b] = lam;
      }
      __syncwarp();
      double nu = 0.0;
      if (e < a.nEl) {
        if (act != (R)0) nu = (double)act * a.avC * a.hEl[e] / (double)N * (double)s.lam[lane];
        a.nu[e] = nu;
        a.act[e] = (float)act;
        if (mlp && a.actInd) a.actInd[e] = (float)actInd;
      }
      const unsigned nzMask = __ballot_sync(0xffffffffu, nu != 0.0);
      if (nzMask) {
        int b0 = 0;
        if (lane == 0) b0 = atomicAdd(a.activeCount, __popc(nzMask));
        b0 = __shfl_sync(0xffffffffu, b0, 0);
        if (nu != 0.0) a.activeList[b0 + __popc(nzMask & ((1u << lane) - 1u))] = (int)e;
      }
      __syncwarp();
    }
  }
}

// ------------------------------------------------------ viscous-term kernel
// The active elements only (the list the viscosity kernel filled): BR1
// gradient scaled by nu, contravariant viscous flux and face traces of nu grad q.
template <int P, typename R>
struct GradSmem {
  static constexpr int PP = P * P;
  R q[4][PP];
  R dsdx[4][PP];  // (dsdx11, dsdx21, dsdx12, dsdx22) per node
  R avg[4][4][P];
  R g[2][4][PP];  // nu grad q
};

template <int P, typename R>
constexpr int av_elems_per_block() {
  int e = 128 / (P * P);
  if (e < 1) e = 1;
  while (e > 1 && (size_t)e * sizeof(GradSmem<P, R>) > 30 * 1024) --e;
  return e;
}

template <int P, typename R, int EPB>
__global__ void __launch_bounds__(EPB* P* P, 4) k_av_grad(const AvArgs a) {
  constexpr int PP = P * P, N = P - 1, VS = visc_side_stride<P>();
  constexpr int TS = trace_side_stride<P, 9, R>();
  __shared__ GradSmem<P, R> sm_all[EPB];
  __shared__ double sdg[PP], sb[2 * P], sw[P];
  const int tid = threadIdx.x;
  const int slot = tid / PP;
  const int t = tid - slot * PP;
  const int i = t % P, j = t / P;
  GradSmem<P, R>& sm = sm_all[slot];
  for (int k = tid; k < PP; k += blockDim.x) sdg[k] = a.dgM[k];
  for (int k = tid; k < 2 * P; k += blockDim.x) sb[k] = a.bM[k];
  for (int k = tid; k < P; k += blockDim.x) sw[k] = a.qw[k];
  __syncthreads();
  const R* trIn = reinterpret_cast<const R*>(a.trIn);
  const int count = *a.activeCount;
  // every block runs the same number of rounds (block-uniform barriers)
  for (int base = blockIdx.x * EPB; base < count; base += gridDim.x * EPB) {
    const bool live = base + slot < count && t < PP;
    const long long e = live ? a.activeList[base + slot] : 0;
    if (live) {
#pragma unroll
      for (int v = 0; v < 4; ++v) sm.q[v][t] = (R)a.q[t + (long long)PP * (v + 4 * e)];
      const double* gd = a.dsdx + 4 * (t + (long long)PP * e);
#pragma unroll
      for (int k = 0; k < 4; ++k) sm.dsdx[k][t] = (R)gd[k];
      // averaged conservative traces (BassiRebaySides) with the stage's exterior states
      for (int k = t; k < 4 * P; k += PP) {
        const int s1 = k / P, ii = k % P;
        const int* si = a.sideInfo + 5 * (s1 + 4 * e);
        const R* own = trIn + (long long)TS * (s1 + 4 * e);
        R L[4], X[4];
#pragma unroll
        for (int w = 0; w < 4; ++w) {
          L[w] = own[ii + P * w];
          X[w] = (R)0;
        }
        const int bcid = si[4];
        if (bcid == 0) {
          const long long e2 = si[2] - 1;
          const int s2 = si[3] / 10 - 1, flip = si[3] % 10;
          const R* nb = trIn + (long long)TS * (s2 + 4 * e2);
          const int i2 = flip ? N - ii : ii;
#pragma unroll
          for (int w = 0; w < 4; ++w) X[w] = nb[i2 + P * w];
        } else if (si[2] == 0) {  // physical side: the boundary condition's exterior state
          if (bcid == SG_BC_NONORMALFLOW) {
            const double2 nh = reinterpret_cast<const double2*>(a.nHat)[ii + (long long)P * (s1 + 4 * e)];
            reflect<R>(L[0], L[1], nh.x, nh.y, X[0], X[1]);
            X[2] = L[2];
            X[3] = L[3];
          } else if ((bcid == SG_BC_PRESCRIBED || bcid == SG_BC_RADIATION) && a.presc) {
#pragma unroll
            for (int w = 0; w < 4; ++w) X[w] = (R)a.presc[ii + (long long)P * (w + 4 * (s1 + 4 * e))];
          }
        }
#pragma unroll
        for (int w = 0; w < 4; ++w) sm.avg[s1][w][ii] = (R)0.5 * (L[w] + X[w]);
      }
    }
    __syncthreads();
    // BR1 gradient (GradientBR_MappedScalar2D, src/SELF_MappedData.f90:990-1074) scaled by nu,
    // and the contravariant viscous flux (src/models/hip/SELF_Advection2D.cpp:66-95)
    if (live) {
      const R nu = (R)a.nu[e];
      const double* nH = a.nHat + 2 * (long long)P * 4 * e;
      const double* nS = a.nScale + (long long)P * 4 * e;
      const R Jij = (R)a.J[t + (long long)PP * e];
      R* visc = reinterpret_cast<R*>(a.visc);
#pragma unroll 1
      for (int v = 0; v < 4; ++v) {
        R gx = (R)0, gy = (R)0;
#pragma unroll
        for (int ii = 0; ii < P; ++ii) {
          const R qa = sm.q[v][ii + P * j], qb = sm.q[v][i + P * ii];
          R f1 = qa * sm.dsdx[0][ii + P * j];
          R f2 = qb * sm.dsdx[2][i + P * ii];
          gx = gx + (R)sdg[ii + P * i] * f1 + (R)sdg[ii + P * j] * f2;
          f1 = qa * sm.dsdx[1][ii + P * j];
          f2 = qb * sm.dsdx[3][i + P * ii];
          gy = gy + (R)sdg[ii + P * i] * f1 + (R)sdg[ii + P * j] * f2;
        }
        // nHat(d, k, side) at nH[d + 2 (k + P side)], nScale(k, side) at nS[k + P side]
        R f1 = sm.avg[1][v][j] * (R)nH[0 + 2 * (j + P * 1)] * (R)nS[j + P * 1];
        R f2 = sm.avg[3][v][j] * (R)nH[0 + 2 * (j + P * 3)] * (R)nS[j + P * 3];
        gx = gx + (f1 * (R)sb[i + P] + f2 * (R)sb[i]) / (R)sw[i];
        f1 = sm.avg[2][v][i] * (R)nH[0 + 2 * (i + P * 2)] * (R)nS[i + P * 2];
        f2 = sm.avg[0][v][i] * (R)nH[0 + 2 * (i + P * 0)] * (R)nS[i + P * 0];
        gx = gx + (f1 * (R)sb[j + P] + f2 * (R)sb[j]) / (R)sw[j];
        f1 = sm.avg[1][v][j] * (R)nH[1 + 2 * (j + P * 1)] * (R)nS[j + P * 1];
        f2 = sm.avg[3][v][j] * (R)nH[1 + 2 * (j + P * 3)] * (R)nS[j + P * 3];
        gy = gy + (f1 * (R)sb[i + P] + f2 * (R)sb[i]) / (R)sw[i];
        f1 = sm.avg[2][v][i] * (R)nH[1 + 2 * (i + P * 2)] * (R)nS[i + P * 2];
        f2 = sm.avg[0][v][i] * (R)nH[1 + 2 * (i + P * 0)] * (R)nS[i + P * 0];
        gy = gy + (f1 * (R)sb[j + P] + f2 * (R)sb[j]) / (R)sw[j];
        gx = gx / Jij;
        gy = gy / Jij;
        gx = gx * nu;
        gy = gy * nu;
        sm.g[0][v][t] = gx;
        sm.g[1][v][t] = gy;
        const R c1 = -(sm.dsdx[0][t] * gx + sm.dsdx[1][t] * gy);
        const R c2 = -(sm.dsdx[2][t] * gx + sm.dsdx[3][t] * gy);
        visc[t + (long long)PP * (0 + 2 * (v + 4 * e))] = c1;
        visc[t + (long long)PP * (1 + 2 * (v + 4 * e))] = c2;
      }
    }
    __syncthreads();
    // face traces of nu grad q (VectorBoundaryInterp_2D, src/SELF_Lagrange.f90:2284-2316)
    if (live) {
      R* vo = reinterpret_cast<R*>(a.vtr) + (long long)4 * VS * e;
      for (int k = t; k < 4 * 8 * P; k += PP) {
        const int ii = k % P, d = (k / P) % 2, v = (k / (2 * P)) % 4, s1 = k / (8 * P);
        vo[s1 * VS + ii + P * (d + 2 * v)] = face_trace<P, R>(sm.g[d][v], sb, s1, ii);
      }
    }
    __syncthreads();  // the slot's arrays are reused by the next round
  }
}

// Closure features of a stored FP64 state (training-data harvest): per element
// the indicator activation and the 36 features.
template <int P>
__global__ void __launch_bounds__(P* P) k_closure_features(const double* __restrict__ q, int nEl, AvArgs a,
                                                            float* __restrict__ act, float* __restrict__ feat) {
  constexpr int PP = P * P;
  __shared__ double sq[2][PP], tt[2][PP], cc[2][PP], sT[PP];
  const int t = threadIdx.x, i = t % P, j = t / P;
  const long long e = blockIdx.x;
  if (e >= nEl) return;
  sT[t] = a.T[t];
  sq[0][t] = q[t + (long long)PP * (2 + 4 * e)];
  sq[1][t] = q[t + (long long)PP * (3 + 4 * e)];
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    double acc = 0.0;
    for (int m = 0; m < P; ++m) acc = acc + sT[i + P * m] * sq[r][m + P * j];
    tt[r][i + P * j] = acc;
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    double acc = 0.0;
    for (int m = 0; m < P; ++m) acc = acc + sT[j + P * m] * tt[r][i + P * m];
    cc[r][i + P * j] = acc;
  }
  __syncthreads();
  if (t == 0 && act) act[e] = (float)modal_activation<P, double>(cc[0], a.s0, a.kappa);
  if constexpr (P >= 6) {
    if (t < 2 && feat) modal_features<P, double>(cc[t], feat + kMlpIn * e + 18 * t);
  }
}

struct QwArr {
  double w[kMaxP];
};

// formNu: form the element viscosity and the active list (the first stage of
// an RK step, or a tendency evaluation); otherwise the viscous terms are
// formed with the viscosity the step's first stage found.
template <int P, typename R>
cudaError_t launch_av_pair(const AvArgs& a, cudaStream_t st, int numSMs, bool formNu) {
  constexpr int EPB = av_elems_per_block<P, R>();
  if (!formNu) {
    k_av_grad<P, R, EPB><<<4 * numSMs, EPB * P * P, 0, st>>>(a);
    return cudaGetLastError();
  }
  cudaError_t e = cudaMemsetAsync(a.activeCount, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  // one wave of resident blocks, each warp striding over its share of the
  // elements (a partial second wave would run at low occupancy)
  static std::atomic<int> nuPerSM{0};  // resident blocks per SM, one instantiation per (P, R)
  if (nuPerSM.load() == 0) {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_av_nu<P, R>, 32 * kNuWarps, 0) != cudaSuccess || nb < 1)
      nb = 4;
    nuPerSM.store(nb);
  }
  const long long nuBlocks = (a.nEl + kNuWarps - 1) / kNuWarps;
  const long long cap = (long long)nuPerSM.load() * numSMs;
  const int g1 = (int)(nuBlocks < cap ? nuBlocks : cap);
  k_av_nu<P, R><<<g1, 32 * kNuWarps, 0, st>>>(a);
  k_av_grad<P, R, EPB><<<4 * numSMs, EPB * P * P, 0, st>>>(a);
  return cudaGetLastError();
}

template <typename R>
cudaError_t launch_av_prep_impl(int P, const AvArgs& a, cudaStream_t st, int numSMs, bool formNu) {
  switch (P) {
    case 2: return launch_av_pair<2, R>(a, st, numSMs, formNu);
    case 3: return launch_av_pair<3, R>(a, st, numSMs, formNu);
    case 4: return launch_av_pair<4, R>(a, st, numSMs, formNu);
    case 5: return launch_av_pair<5, R>(a, st, numSMs, formNu);
    case 6: return launch_av_pair<6, R>(a, st, numSMs, formNu);
    case 7: return launch_av_pair<7, R>(a, st, numSMs, formNu);
    case 8: return launch_av_pair<8, R>(a, st, numSMs, formNu);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace selfgpu
