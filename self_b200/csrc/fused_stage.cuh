// Fused DGSEM stage kernels: one launch per low-storage RK stage.
//
// Per element and per stage m they do everything CalculateTendency_Model2D +
// UpdateGRK3_Model2D do (src/SELF_Model2D.f90:816-859, :710-752):
//
//   1. stage the element's solution, form the point-wise auxiliaries
//      (CIG: u, v, p, rhoH, c; SW: u, v) and the contravariant volume flux
//      F~1 = dsdx(1,1)Fx + dsdx(2,1)Fy,  F~2 = dsdx(1,2)Fx + dsdx(2,2)Fy;
//   2. interpolate the element's own face traces (BoundaryInterp) and take the
//      neighbours' traces of the same stage from the trace cache written by the
//      previous launch (SideExchange, flip applied on the fly); physical sides
//      get their exterior state from the model's boundary condition;
//   3. Riemann flux at the 4P face nodes, already scaled by nScale;
//   4. weak divergence with surface lift and the 1/J weighting
//      (VectorDGDivergence_2D + JacobianWeight), dSdt = source - div;
//   5. G = a_m G + dSdt,  q = q + (g_m dt) G  in place (FP64);
//   6. interpolate the traces of the updated solution and write them to the
//      other half of the ping-pong trace cache for the next launch.
//
// Global traffic per element-stage is the algorithmic minimum for a stage with
// one face exchange: solution and G read+write, metric terms read once, own
// traces written once, neighbour traces read once.
//
// Two kernels implement this: k_fused_stage (below; one CTA of P*P-thread
// element groups, plain loads; any degree) and k_fused_stage_tma
// (fused_stage_tma.cuh; persistent, bulk-async copies into a shared-memory
// ring; even P).  Both share the model policies and the trace-cache layout.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "physics.cuh"

namespace selfgpu {

constexpr int kMaxP = 8;

enum StageMode { MODE_TRACES = 0, MODE_TENDENCY = 1, MODE_RK = 2 };

struct StageArgs {
  int nEl;
  int mode;
  // geometry (caller owned, FP64)
  const double* __restrict__ dsdx;    // (2,2,P,P,1,nEl)
  const double* __restrict__ J;       // (P,P,1,nEl)
  const double* __restrict__ nHat;    // (2,P,1,4,nEl)
  const double* __restrict__ nScale;  // (P,1,4,nEl)
  const int* __restrict__ sideInfo;   // (5,4,nEl)
  // state (caller owned, FP64)
  double* q;     // (P,P,NV,nEl)
  double* G;     // (P,P,NV,nEl) RK register (FP64 forms)
  float* Gf;     // (P,P,NV,nEl) RK register of the FP32-bulk form (engine owned; G is then unused)
  double* dSdt;  // (P,P,NV,nEl), MODE_TENDENCY only
  // engine-owned trace cache (bulk type): per (element, side) a block of TS
  // values holding NT fields x P nodes, padded to 16 bytes
  const void* trIn;
  void* trOut;
  // ShallowWater stage-lagged velocity traces (P, 2, 4, nEl), bulk type
  const void* velIn;
  void* velOut;
  // model parameters and fields (FP64, caller owned; NULL = absent)
  double g, fC, gamma, Rgas;
  const double* fld[5];
  // RK coefficients: G = a G + dSdt ; q = q + gdt G, with gdt = rk_gdt, or
  // rk_g * dtElem[e] when a per-element time step is bound (ensembles)
  double rk_a, rk_gdt, rk_g;
  const double* dtElem;
  // artificial-viscosity closure (CIG; av_closure.cuh): contravariant viscous
  // volume flux (P*P, 2, 4, nEl) and per (element, side) face traces of
  // nu grad q (8P values at [i + P (d + 2 v)]), both bulk type
  int av;
  const void* visc;
  const void* vtr;
  const double* avNu;  // element viscosity: elements with nu = 0 have no viscous terms
  // engine-owned packed geometry: per element one contiguous record of
  // geo_rec(P, kind).bytes (dsdx, nHat, nScale, J or 1/J, sideInfo; the kind
  // follows the form); read by the persistent kernel with one bulk copy
  const double* geo;
  // bounded waits of the persistent kernel (clock cycles) and its error word
  long long waitCycles;
  int* err;
  int debugStarve;  // test hooks: 1 = the first element of CTA 0 is registered on its mbarrier but never
                    // copied; 2 = (multi-stage launch) group 0 of CTA 0 never announces a stage end
  // operator matrices (Lagrange%Init): dgM(ii,i) at [ii + P*i], bM(ii,side), qw;
  // bMf holds bM rounded to float for the FP32-bulk form
  double dgM[kMaxP * kMaxP];
  double bM[2 * kMaxP];
  double qw[kMaxP];
  float bMf[2 * kMaxP];
};

// Boundary interpolation weights of the left (S, W) and right (E, N) ends as
// kernel-parameter constants (compile-time index m after unrolling).
template <typename R>
__device__ __forceinline__ R bm_left(const StageArgs& a, int m) {
  if constexpr (sizeof(R) == 8) return a.bM[m];
  else return a.bMf[m];
}
template <typename R, int P>
__device__ __forceinline__ R bm_right(const StageArgs& a, int m) {
  if constexpr (sizeof(R) == 8) return a.bM[m + P];
  else return a.bMf[m + P];
}

// One element's packed geometry record: dsdx (4 P^2 values, as two planes of
// P^2 pairs: (dsdx11, dsdx21) of every node, then (dsdx12, dsdx22)), nHat
// (8 P), nScale (4 P), a J slot (P^2 doubles), sideInfo (20 ints).  Four kinds:
//   GEO_REF   FP64 metrics, J            (reference-rounding form)
//   GEO_INVJ  FP64 metrics, 1/J          (production FP64 at P != 8)
//   GEO_NOJ   FP64 metrics, no J slot    (production FP64 at P = 8: the stage
//             takes 1/J as the reciprocal of det(dsdx) = J, dsdx being the
//             adjugate of the covariant basis)
//   GEO_F32   FP32 metrics, FP64 1/J     (FP32 bulk: its stage rounds dsdx,
//             nHat and nScale to FP32 before every use, so the record holds
//             them rounded once; 1/J stays FP64)
// Every kind is a multiple of 16 bytes for even P.
enum GeoKind { GEO_REF = 0, GEO_INVJ = 1, GEO_NOJ = 2, GEO_F32 = 3 };
struct GeoRec {
  int wm;                                // bytes per metric value (8 or 4)
  int oNhat, oNs, oJ, oSi, bytes;        // byte offsets within a record, record size
};
__host__ __device__ constexpr GeoRec geo_rec(int P, int kind) {
  const int wm = kind == GEO_F32 ? 4 : 8;
  const int oNhat = 4 * P * P * wm, oNs = oNhat + 8 * P * wm, oJ = oNs + 4 * P * wm;
  const int oSi = oJ + (kind == GEO_NOJ ? 0 : 8 * P * P);
  return GeoRec{wm, oNhat, oNs, oJ, oSi, oSi + 80};
}

// Trace-cache block size (values of the bulk type) of one (element, side).
template <int P, int NT, typename R>
__host__ __device__ constexpr int trace_side_stride() {
  constexpr int per16 = 16 / (int)sizeof(R);
  return (NT * P + per16 - 1) / per16 * per16;
}

// ---------------------------------------------------------------- policies
// NV state variables, NT traced fields, NF per-node fields kept in smem.
// Node aux a[3] and face aux x[9] are fetched by the kernel:
//   LSW  a = (H, fCori)            x = (H.boundary)
//   SW   a = (dh/dx, dh/dy)        x = (topography.boundary)
//   CIG  a = (gx, gy, Cd)          x = prescribed (rhoU,rhoV,rho,rhoE,u,v,p,rhoH,c)
inline namespace SELFGPU_FORM_NS {

// The record kind a stage kernel of bulk type R reads at P.
template <int P, typename R>
__host__ __device__ constexpr int geo_kind() {
  return (sizeof(R) == 4) ? GEO_F32
         : ref_rounding<R>()                   ? GEO_REF
         : (P == 8 ? GEO_NOJ : GEO_INVJ);
}

struct PhysLSW {
  static constexpr int NV = 3, NT = 3, NF = 3;
  static constexpr bool kLaggedVelocity = false;
  template <typename R>
  __device__ static void node(R*, const StageArgs&) {}
  template <typename R>
  __device__ static void node_flux(R*, const StageArgs&) {}
  template <typename R>
  __device__ static void flux(const R* f, const double* a, const StageArgs& s, R Fx[3], R Fy[3]) {
    const R H = (R)a[0], g = (R)s.g;  // src/models/SELF_LinearShallowWater.f90:470-490
    Fx[0] = g * f[2];
    Fy[0] = (R)0;
    Fx[1] = (R)0;
    Fy[1] = g * f[2];
    Fx[2] = H * f[0];
    Fy[2] = H * f[1];
  }
  template <typename R>
  __device__ static void source(const R* f, const double* a, const StageArgs&, R S[3]) {
    const R fc = (R)a[1];  // src/models/SELF_LinearShallowWater.f90:433-439
    S[0] = fc * f[1];
    S[1] = -fc * f[0];
    S[2] = (R)0;
  }
  template <typename R>
  __device__ static void face(int bcid, bool physical, const R* L, R* X, const R*, const R*, double n1, double n2,
                              double nmag, const double* x, const StageArgs& s, R out[3]) {
    if (physical) {  // src/models/SELF_LinearShallowWater.f90:323-349
      if (bcid == SG_BC_NONORMALFLOW) {
        reflect<R>(L[0], L[1], n1, n2, X[0], X[1]);
        X[2] = L[2];
      } else {
        X[0] = X[1] = X[2] = (R)0;
      }
    }
    lsw_riemann<R>(L[0], L[1], L[2], X[0], X[1], X[2], (R)x[0], (R)s.g, n1, n2, nmag, out);
  }
};

struct PhysSW {
  static constexpr int NV = 3, NT = 3, NF = 5;
  static constexpr bool kLaggedVelocity = true;
  template <typename R>
  __device__ static void node(R* f, const StageArgs&) {
    const R H = f[2];  // src/models/SELF_ShallowWater.f90:205-216
    if constexpr (ref_rounding<R>()) {
      f[3] = f[0] / H;
      f[4] = f[1] / H;
    } else {
      const R r = (R)1 / H;
      f[3] = f[0] * r;
      f[4] = f[1] * r;
    }
  }
  template <typename R>
  __device__ static void node_flux(R* f, const StageArgs& s) {
    node<R>(f, s);
  }
  template <typename R>
  __device__ static void flux(const R* f, const double*, const StageArgs& s, R Fx[3], R Fy[3]) {
    sw_flux<R>(f[0], f[1], f[2], f[3], f[4], (R)s.g, Fx, Fy);
  }
  template <typename R>
  __device__ static void source(const R* f, const double* a, const StageArgs& s, R S[3]) {
    const R g = (R)s.g, fc = (R)s.fC;  // src/models/SELF_ShallowWater.f90:362-378
    S[0] = -fc * f[1] + g * f[2] * (R)a[0];
    S[1] = fc * f[0] + g * f[2] * (R)a[1];
    S[2] = (R)0;
  }
  template <typename R>
  __device__ static void face(int bcid, bool physical, const R* L, R* X, const R* velL, const R* velR, double n1,
                              double n2, double nmag, const double* x, const StageArgs& s, R out[3]) {
    if (physical) {  // src/models/SELF_ShallowWater.f90:305-338
      if (bcid == SG_BC_NONORMALFLOW) {
        reflect<R>(L[0], L[1], n1, n2, X[0], X[1]);
        X[2] = L[2];
      } else {
        X[0] = X[1] = (R)0;
        X[2] = (R)x[0];
      }
    }
    sw_riemann<R>(L[0], L[1], L[2], X[0], X[1], X[2], velL[0], velL[1], velR[0], velR[1], (R)s.g, n1, n2, nmag, out);
  }
};

struct PhysCIG {
  static constexpr int NV = 4, NT = 9, NF = 9;
  static constexpr bool kLaggedVelocity = false;
  // The primitive and diagnostic traces are interpolated fields, not
  // recomputed from interpolated conservative traces (src/models/
  // SELF_CompressibleIdealGas2D.f90:972-980).
  template <typename R>
  __device__ static void node(R* f, const StageArgs& s) {
    R u, v, p, ke, h, c;
    cig_state<R>(f[0], f[1], f[2], f[3], (R)s.gamma, u, v, p, ke, h, c);
    f[4] = u;
    f[5] = v;
    f[6] = p;
    f[7] = h;
    f[8] = c;
  }
  // The volume flux needs u, v, p and rhoH only (no sound speed).
  template <typename R>
  __device__ static void node_flux(R* f, const StageArgs& s) {
    R u, v;
    if constexpr (!ref_rounding<R>()) {  // FP32 bulk / production FP64: one reciprocal of the density
      const R r = (R)1 / f[2];
      u = f[0] * r;
      v = f[1] * r;
    } else {
      u = f[0] / f[2];
      v = f[1] / f[2];
    }
    const R ke = (R)0.5 * (f[0] * u + f[1] * v);
    const R p = ((R)s.gamma - (R)1) * (f[3] - ke);
    f[4] = u;
    f[5] = v;
    f[6] = p;
    f[7] = f[3] + p;
  }
  template <typename R>
  __device__ static void flux(const R* f, const double*, const StageArgs&, R Fx[4], R Fy[4]) {
    cig_flux<R>(f[0], f[1], f[4], f[5], f[6], f[7], Fx, Fy);
  }
  template <typename R>
  __device__ static void source(const R* f, const double* a, const StageArgs&, R S[4]) {
    const R gx = (R)a[0], gy = (R)a[1], cd = (R)a[2];  // src/models/SELF_CompressibleIdealGas2D.f90:1339-1360
    S[0] = -f[2] * gx - cd * f[0];
    S[1] = -f[2] * gy - cd * f[1];
    S[2] = (R)0;
    S[3] = -f[0] * gx - f[0] * gy;
  }
  template <typename R>
  __device__ static void face(int bcid, bool physical, const R* L, R* X, const R*, const R*, double n1, double n2,
                              double nmag, const double* x, const StageArgs& s, R out[4]) {
    if (physical) {  // src/models/SELF_CompressibleIdealGas2D.f90:1256-1317
      if (bcid == SG_BC_NONORMALFLOW) {
        reflect<R>(L[0], L[1], n1, n2, X[0], X[1]);
        X[2] = L[2];
        X[3] = L[3];
        reflect<R>(L[4], L[5], n1, n2, X[4], X[5]);
        X[6] = L[6];
        X[7] = L[7];
        X[8] = L[8];
      } else if ((bcid == SG_BC_PRESCRIBED || bcid == SG_BC_RADIATION) && s.fld[2] != nullptr) {
        for (int k = 0; k < 9; ++k) X[k] = (R)x[k];
      } else {
        for (int k = 0; k < 9; ++k) X[k] = (R)0;
      }
    }
    cig_llf<R>(L, X, n1, n2, nmag, out);
  }
};

}  // namespace SELFGPU_FORM_NS

// Model fields from global memory (v1 kernel).  t = node, e = element.
template <class Phys>
__device__ __forceinline__ void node_aux_global(const StageArgs& s, int t, long long e, int PP, double a[3]) {
  a[0] = a[1] = a[2] = 0.0;
  const long long gn = t + (long long)PP * e;
  if constexpr (Phys::NV == 3 && !Phys::kLaggedVelocity) {  // LSW
    a[0] = s.fld[0][gn];
    if (s.fld[2]) a[1] = s.fld[2][gn];
  } else if constexpr (Phys::kLaggedVelocity) {  // SW
    if (s.fld[1]) {
      a[0] = s.fld[1][2 * gn];
      a[1] = s.fld[1][2 * gn + 1];
    }
  } else {  // CIG: environmentalsGradient variable 1, environmentals variable 2
    if (s.fld[0]) {
      const double* gg = s.fld[0] + 2 * (t + (long long)PP * 2 * e);
      a[0] = gg[0];
      a[1] = gg[1];
    }
    if (s.fld[1]) a[2] = s.fld[1][t + (long long)PP * (1 + 2 * e)];
  }
}

template <class Phys>
__device__ __forceinline__ void face_aux_global(const StageArgs& s, int side, int i, long long e, int P, double x[9]) {
  const long long gf = i + (long long)P * (side + 4 * e);
  if constexpr (Phys::NV == 3 && !Phys::kLaggedVelocity) {
    x[0] = s.fld[1][gf];
  } else if constexpr (Phys::kLaggedVelocity) {
    x[0] = s.fld[0] ? s.fld[0][gf] : 0.0;
  } else {
    if (s.fld[2]) {
      const long long b = i + (long long)P * 4 * (side + 4 * e);  // (i, var, side, el), 4 vars
      for (int v = 0; v < 4; ++v) x[v] = s.fld[2][b + v * P];
      x[4] = s.fld[3][b];
      x[5] = s.fld[3][b + P];
      x[6] = s.fld[3][b + 3 * P];
      x[7] = s.fld[4][b + P];
      x[8] = s.fld[4][b + 2 * P];
    }
  }
}

// Viscous closure terms (CompressibleIdealGas2D only).  Volume: the
// contravariant viscous flux is added to the contravariant inviscid flux.
// Face: on exchanged sides -1/2 (nu grad q_in + nu grad q_ex) . n nScale is
// added to the Riemann flux, the exterior value taken from the neighbour's
// traces with the flip applied (src/models/hip/SELF_Advection2D.cpp:140-175
// with one viscosity per element); physical sides carry no viscous flux.
template <int P>
__host__ __device__ constexpr int visc_side_stride() {
  return 8 * P;  // 2 components x 4 variables x P nodes
}

template <int P, typename R>
__device__ __forceinline__ void av_volume_add(const StageArgs& s, int t, long long e, R* F0, R* F1) {
  constexpr int PP = P * P;
  if (s.avNu[e] == 0.0) return;
  const R* vs = reinterpret_cast<const R*>(s.visc) + t + (long long)PP * 8 * e;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    F0[v] = F0[v] + vs[PP * (0 + 2 * v)];
    F1[v] = F1[v] + vs[PP * (1 + 2 * v)];
  }
}

template <int P, typename R>
__device__ __forceinline__ void av_face_add(const StageArgs& s, int s1, int ii, long long e, const int* si,
                                            double n1, double n2, double nmag, R out[4]) {
  constexpr int VS = visc_side_stride<P>(), N = P - 1;
  const R* vt = reinterpret_cast<const R*>(s.vtr);
  if (si[4] != 0) return;
  const long long e2 = si[2] - 1;
  const bool aOwn = s.avNu[e] != 0.0, aExt = s.avNu[e2] != 0.0;
  if (!aOwn && !aExt) return;
  const R* own = vt + (long long)VS * (s1 + 4 * e);
  const R* ext = vt + (long long)VS * (si[3] / 10 - 1 + 4 * e2);
  const int ie = (si[3] % 10) ? N - ii : ii;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const R in = aOwn ? own[ii + P * (0 + 2 * v)] * (R)n1 + own[ii + P * (1 + 2 * v)] * (R)n2 : (R)0;
    const R ex = aExt ? ext[ie + P * (0 + 2 * v)] * (R)n1 + ext[ie + P * (1 + 2 * v)] * (R)n2 : (R)0;
    out[v] = out[v] + (R)(-0.5) * (in + ex) * (R)nmag;
  }
}

// Boundary interpolation of one traced field at face node ii of side s1
// (src/SELF_Lagrange.f90:2241-2270): S and N run along j at fixed i, E and W
// along i at fixed j.
template <int P, typename R>
__device__ __forceinline__ R face_trace(const R* fv, const double* sb, int s1, int ii) {
  R acc = (R)0;
  if (s1 == 0) {
#pragma unroll
    for (int m = 0; m < P; ++m) acc = acc + (R)sb[m] * fv[ii + P * m];
  } else if (s1 == 1) {
#pragma unroll
    for (int m = 0; m < P; ++m) acc = acc + (R)sb[m + P] * fv[m + P * ii];
  } else if (s1 == 2) {
#pragma unroll
    for (int m = 0; m < P; ++m) acc = acc + (R)sb[m + P] * fv[ii + P * m];
  } else {
#pragma unroll
    for (int m = 0; m < P; ++m) acc = acc + (R)sb[m] * fv[m + P * ii];
  }
  return acc;
}

// ------------------------------------------------------------- v1 kernel
template <int P, class Phys, typename R>
struct Smem {
  static constexpr int NV = Phys::NV, NT = Phys::NT, NF = Phys::NF, PP = P * P;
  R fld[NF][PP];
  R Fc[2][NV][PP];
  R own[4][NT][P];
  R ext[4][NT][P];
  R fb[4][NV][P];
  R vel[Phys::kLaggedVelocity ? 2 : 1][4][2][P];
};

// The per-stage part of a launch (mode, RK coefficients, the trace-cache
// halves read and written); everything else comes from StageArgs.
struct StageVar {
  int mode;
  double rk_a, rk_gdt, rk_g;
  const void* trIn;
  void* trOut;
  const void* velIn;
  void* velOut;
};

// A load from the trace cache.  kCoherent = true (the multi-stage kernel,
// where other CTAs of the same launch wrote the data a grid barrier ago)
// reads through L2 only, never a possibly stale L1 line.
template <bool kCoherent, typename R>
__device__ __forceinline__ R ld_trace(const R* p) {
  if constexpr (kCoherent) return __ldcg(p);
  else return *p;
}

// One stage over the CTA's EPB element slots (one thread per node): the body
// of k_fused_stage, shared with the multi-stage kernel k_fused_steps.  The
// operator matrices are already in shared memory (sdg, sb, srw).
template <int P, class Phys, typename R, int EPB, bool kCoherent>
__device__ __forceinline__ void fused_stage_group(const StageArgs& a, const StageVar& sv, Smem<P, Phys, R>* sm_all,
                                                  const double* sdg, const double* sb, const double* srw) {
  constexpr int NV = Phys::NV, NT = Phys::NT, NF = Phys::NF, PP = P * P, N = P - 1;
  constexpr int TS = trace_side_stride<P, NT, R>();
  using S = Smem<P, Phys, R>;

  const int tid = threadIdx.x;
  const int slot = tid / PP;
  const int t = tid - slot * PP;  // node index ij = i + P*j
  const int i = t % P, j = t / P;
  S& sm = sm_all[slot];

  const long long e = (long long)blockIdx.x * EPB + slot;
  const bool live = e < a.nEl;
  const R* trIn = reinterpret_cast<const R*>(sv.trIn);
  R* trOut = reinterpret_cast<R*>(sv.trOut);
  const long long gnode = t + (long long)PP * e;

  if (live) {
    R f[NF];
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = (R)a.q[t + (long long)PP * (v + NV * e)];
    Phys::template node<R>(f, a);
#pragma unroll
    for (int v = 0; v < NF; ++v) sm.fld[v][t] = f[v];
    if (sv.mode != MODE_TRACES) {
      double na[3];
      node_aux_global<Phys>(a, t, e, PP, na);
      R Fx[NV], Fy[NV];
      Phys::template flux<R>(f, na, a, Fx, Fy);
      const double2* gp = reinterpret_cast<const double2*>(a.dsdx + 4 * gnode);
      const double2 c1 = gp[0], c2 = gp[1];  // (dsdx11, dsdx21), (dsdx12, dsdx22)
      R F0[NV], F1[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        F0[v] = (R)c1.x * Fx[v] + (R)c1.y * Fy[v];
        F1[v] = (R)c2.x * Fx[v] + (R)c2.y * Fy[v];
      }
      if constexpr (NV == 4)
        if (a.av) av_volume_add<P, R>(a, t, e, F0, F1);
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        sm.Fc[0][v][t] = F0[v];
        sm.Fc[1][v][t] = F1[v];
      }
      for (int k = t; k < 4 * NT * P; k += PP) {
        const int ii = k % P, fs = k / P, fi = fs % NT, s1 = fs / NT;
        const int* si = a.sideInfo + 5 * (s1 + 4 * e);
        R val = (R)0;
        if (si[4] == 0) {
          const long long e2 = si[2] - 1;
          const int s2 = si[3] / 10 - 1, flip = si[3] % 10;
          val = ld_trace<kCoherent>(trIn + (flip ? N - ii : ii) + P * fi + (long long)TS * (s2 + 4 * e2));
        }
        sm.ext[s1][fi][ii] = val;
        // own traces of this stage's solution: the trace cache holds them (the
        // previous launch formed them from the same values with the same sums)
        sm.own[s1][fi][ii] = ld_trace<kCoherent>(trIn + ii + P * fi + (long long)TS * (s1 + 4 * e));
      }
      if constexpr (Phys::kLaggedVelocity) {
        const R* vIn = reinterpret_cast<const R*>(sv.velIn);
        for (int k = t; k < 16 * P; k += PP) {
          const int ii = k % P, d = (k / P) % 2, s1 = (k / (2 * P)) % 4, which = k / (8 * P);
          R val = (R)0;
          if (which == 0) {
            val = ld_trace<kCoherent>(vIn + ii + P * (d + 2 * (s1 + 4 * e)));
          } else {
            const int* si = a.sideInfo + 5 * (s1 + 4 * e);
            if (si[4] == 0) {  // velocity%extBoundary is only ever set by the exchange (H8)
              const long long e2 = si[2] - 1;
              const int s2 = si[3] / 10 - 1, flip = si[3] % 10;
              val = ld_trace<kCoherent>(vIn + (flip ? N - ii : ii) + P * (d + 2 * (s2 + 4 * e2)));
            }
          }
          sm.vel[which][s1][d][ii] = val;
        }
      }
    }
  }
  if (sv.mode != MODE_TRACES) {
    __syncthreads();
    // 4P face nodes per element; for P <= 3 there are fewer node threads (P*P)
    if (live)
      for (int k = t; k < 4 * P; k += PP) {
        const int s1 = k / P, ii = k % P;
        const int* si = a.sideInfo + 5 * (s1 + 4 * e);
        const int bcid = si[4];
        const bool physical = (bcid != 0) && (si[2] == 0);
        R L[NT], X[NT];
#pragma unroll
        for (int m = 0; m < NT; ++m) {
          L[m] = sm.own[s1][m][ii];
          X[m] = (bcid == 0) ? sm.ext[s1][m][ii] : (R)0;
        }
        const long long gface = ii + (long long)P * (s1 + 4 * e);
        const double2 nh = reinterpret_cast<const double2*>(a.nHat)[gface];
        const double ns = a.nScale[gface];
        double fx[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        if (physical) face_aux_global<Phys>(a, s1, ii, e, P, fx);
        else if constexpr (Phys::NV == 3 && !Phys::kLaggedVelocity) face_aux_global<Phys>(a, s1, ii, e, P, fx);
        R velL[2] = {(R)0, (R)0}, velR[2] = {(R)0, (R)0};
        if constexpr (Phys::kLaggedVelocity) {
          velL[0] = sm.vel[0][s1][0][ii];
          velL[1] = sm.vel[0][s1][1][ii];
          velR[0] = sm.vel[1][s1][0][ii];
          velR[1] = sm.vel[1][s1][1][ii];
          R* vOut = reinterpret_cast<R*>(sv.velOut);  // read by the next stage
          vOut[ii + P * (0 + 2 * (s1 + 4 * e))] = L[0] / L[2];
          vOut[ii + P * (1 + 2 * (s1 + 4 * e))] = L[1] / L[2];
        }
        R out[NV];
        Phys::template face<R>(bcid, physical, L, X, velL, velR, nh.x, nh.y, ns, fx, a, out);
        if constexpr (NV == 4)
          if (a.av) av_face_add<P, R>(a, s1, ii, e, si, nh.x, nh.y, ns, out);
#pragma unroll
        for (int v = 0; v < NV; ++v) sm.fb[s1][v][ii] = out[v];
      }
    __syncthreads();
    if (live) {
      R f[NF];
#pragma unroll
      for (int v = 0; v < NF; ++v) f[v] = sm.fld[v][t];
      double na[3];
      node_aux_global<Phys>(a, t, e, PP, na);
      // sources in FP64 in every form (well-balanced topography / gravity terms)
      double qd[NV], Src[NV];
#pragma unroll
      for (int v = 0; v < NV; ++v) qd[v] = a.q[t + (long long)PP * (v + NV * e)];
      Phys::template source<double>(qd, na, a, Src);
      const double Jij = a.J[gnode];
      const R wi = (R)srw[i], wj = (R)srw[j];
      // FP32 bulk and production FP64: products with the reciprocals (the
      // reference-rounding FP64 build divides as the reference does)
      const R rwi = (R)(1.0 / srw[i]), rwj = (R)(1.0 / srw[j]);
      const double rJ = 1.0 / Jij;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        R d = (R)0;
#pragma unroll
        for (int m = 0; m < P; ++m)
          d = d + (R)sdg[m + P * i] * sm.Fc[0][v][m + P * j] + (R)sdg[m + P * j] * sm.Fc[1][v][i + P * m];
        const R lx = (R)sb[i + P] * sm.fb[1][v][j] + (R)sb[i] * sm.fb[3][v][j];
        const R ly = (R)sb[j + P] * sm.fb[2][v][i] + (R)sb[j] * sm.fb[0][v][i];
        double dsdt;
        if constexpr (ref_rounding<R>()) {
          d = d + lx / wi + ly / wj;
          dsdt = Src[v] - (double)d / Jij;
        } else {
          d = d + lx * rwi + ly * rwj;
          dsdt = Src[v] - (double)d * rJ;
        }
        const long long gi = t + (long long)PP * (v + NV * e);
        if (sv.mode == MODE_TENDENCY) {
          a.dSdt[gi] = dsdt;
        } else {
          // the FP32-bulk form carries the RK register in FP32; the solution
          // update below uses this stage's unrounded FP64 value
          const double Gn = sv.rk_a * (sizeof(R) == 4 ? (double)a.Gf[gi] : a.G[gi]) + dsdt;
          if constexpr (sizeof(R) == 4) a.Gf[gi] = (float)Gn;
          else a.G[gi] = Gn;
          const double qn = qd[v] + (a.dtElem ? sv.rk_g * a.dtElem[e] : sv.rk_gdt) * Gn;
          a.q[gi] = qn;
          f[v] = (R)qn;
        }
      }
      if (sv.mode == MODE_RK) {
        // only this thread reads node t of fld in this phase, so it may overwrite it
        Phys::template node<R>(f, a);
#pragma unroll
        for (int v = 0; v < NF; ++v) sm.fld[v][t] = f[v];
      }
    }
    if (sv.mode == MODE_TENDENCY) return;
  }
  __syncthreads();
  // traces of the (updated) solution -> trace cache: one task per (field,
  // line, orientation) forms both end traces of the line (column l: S and N,
  // row l: W and E) with the bMatrix rows as kernel-parameter constants
  R* o = trOut + (long long)4 * TS * e;
  if (live)
    for (int k = t; k < 2 * NT * P; k += PP) {
      const int fi = k / (2 * P), rem = k - fi * 2 * P, row = rem / P, l = rem - row * P;
      const R* fv = sm.fld[fi] + (row ? P * l : l);
      const int stride = row ? 1 : P;
      R lo = (R)0, hi = (R)0;
#pragma unroll
      for (int m = 0; m < P; ++m) {
        const R x = fv[stride * m];
        lo = lo + bm_left<R>(a, m) * x;
        hi = hi + bm_right<R, P>(a, m) * x;
      }
      o[l + P * fi + TS * (row ? 3 : 0)] = lo;
      o[l + P * fi + TS * (row ? 1 : 2)] = hi;
    }
  if constexpr (Phys::kLaggedVelocity) {
    // Start of a run: the stage-lagged velocity traces equal those of this
    // solution (SetSolution leaves solution%boundary = BoundaryInterp(solution)).
    if (sv.mode == MODE_TRACES && sv.velOut != nullptr) {
      __syncthreads();
      if (live)
        for (int k = t; k < 4 * P; k += PP) {
          const int s1 = k / P, ii = k % P;
          R* vOut = reinterpret_cast<R*>(sv.velOut);
          const R H = o[ii + P * 2 + TS * s1];
          vOut[ii + P * (0 + 2 * (s1 + 4 * e))] = o[ii + P * 0 + TS * s1] / H;
          vOut[ii + P * (1 + 2 * (s1 + 4 * e))] = o[ii + P * 1 + TS * s1] / H;
        }
    }
  }
}


template <int P, class Phys, typename R, int EPB>
__global__ void __launch_bounds__(EPB* P* P) k_fused_stage(const StageArgs a) {
  constexpr int PP = P * P;
  __shared__ Smem<P, Phys, R> sm_all[EPB];
  __shared__ double sdg[PP], sb[2 * P], srw[P];
  for (int k = threadIdx.x; k < PP; k += blockDim.x) sdg[k] = a.dgM[k];
  for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) sb[k] = a.bM[k];
  for (int k = threadIdx.x; k < P; k += blockDim.x) srw[k] = a.qw[k];
  const StageVar sv{a.mode, a.rk_a, a.rk_gdt, a.rk_g, a.trIn, a.trOut, a.velIn, a.velOut};
  fused_stage_group<P, Phys, R, EPB, false>(a, sv, sm_all, sdg, sb, srw);
}

// ------------------------------------------------- multi-stage (one launch)
// Arguments of k_fused_steps: nSteps Williamson RK3 steps of size dt from
// the trace-cache halves cur / vcur, with a grid barrier counter.
struct StepsArgs {
  int nSteps;
  double dt;
  double rkA[3], rkG[3];
  const void* tr[2];
  const void* vel[2];
  int cur, vcur;
  unsigned* bar;  // zero at launch; counts CTA arrivals over all barriers
};

// Grid-wide barrier number k (1-based) of a launch whose CTAs are all
// resident (cooperative launch).  Bounded: a CTA that waits longer than
// `cycles` sets the error word and returns false (the launch then stops).
__device__ __forceinline__ bool grid_barrier(unsigned* bar, unsigned k, long long cycles, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(bar, 1u);
    const unsigned target = k * gridDim.x;
    int ok = 1;
    const long long t0 = clock64();
    while (true) {
      unsigned v;
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
      if (v >= target) break;
      if (clock64() - t0 > cycles) {
        ok = 0;
        if (err) atomicExch(err, 1);
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// All RK stages of nSteps steps in one cooperative launch, for meshes whose
// element groups fit one wave of resident CTAs (the small, launch-latency
// bound cases): each stage is the k_fused_stage body over the CTA's elements,
// then a grid barrier before the next stage reads the traces other CTAs
// wrote.  Trace reads go through L2 (ld_trace<true>).
template <int P, class Phys, typename R, int EPB>
__global__ void __launch_bounds__(EPB* P* P) k_fused_steps(const StageArgs a, const StepsArgs sa) {
  constexpr int PP = P * P;
  __shared__ Smem<P, Phys, R> sm_all[EPB];
  __shared__ double sdg[PP], sb[2 * P], srw[P];
  for (int k = threadIdx.x; k < PP; k += blockDim.x) sdg[k] = a.dgM[k];
  for (int k = threadIdx.x; k < 2 * P; k += blockDim.x) sb[k] = a.bM[k];
  for (int k = threadIdx.x; k < P; k += blockDim.x) srw[k] = a.qw[k];
  int cur = sa.cur, vcur = sa.vcur;
  unsigned k = 0;
  for (int s = 0; s < sa.nSteps; ++s)
    for (int m = 0; m < 3; ++m) {
      StageVar sv;
      sv.mode = MODE_RK;
      sv.rk_a = sa.rkA[m];
      sv.rk_gdt = sa.rkG[m] * sa.dt;
      sv.rk_g = sa.rkG[m];
      sv.trIn = sa.tr[cur];
      sv.trOut = const_cast<void*>(sa.tr[1 - cur]);
      sv.velIn = sa.vel[vcur];
      sv.velOut = const_cast<void*>(sa.vel[1 - vcur]);
      fused_stage_group<P, Phys, R, EPB, true>(a, sv, sm_all, sdg, sb, srw);
      cur ^= 1;
      if constexpr (Phys::kLaggedVelocity) vcur ^= 1;
      if (!grid_barrier(sa.bar, ++k, a.waitCycles, a.err)) return;
    }
}

}  // namespace selfgpu
