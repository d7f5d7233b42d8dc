// Fused DGSEM stage kernel: one launch per low-storage RK stage.
//
// Per element (one group of P*P threads, one thread per node (i,j)) and per
// stage m it does everything CalculateTendency_Model2D + UpdateGRK3_Model2D do
// (src/SELF_Model2D.f90:816-859, :710-752):
//
//   1. stage the element's solution in shared memory, form the point-wise
//      auxiliaries (CIG: u, v, p, rhoH, c; SW: u, v) and the contravariant
//      volume flux  F~1 = dsdx(1,1)Fx + dsdx(2,1)Fy,  F~2 = dsdx(1,2)Fx + dsdx(2,2)Fy;
//   2. interpolate the element's own face traces (BoundaryInterp) and fetch the
//      neighbours' traces of the same stage from the trace cache written by the
//      previous launch (SideExchange, flip applied on the fly); physical sides
//      get their exterior state from the model's boundary condition;
//   3. Riemann flux at the 4P face nodes, already scaled by nScale;
//   4. weak divergence with surface lift and the 1/J division
//      (VectorDGDivergence_2D + JacobianWeight), dSdt = source - div;
//   5. G = a_m G + dSdt,  q = q + (g_m dt) G  in place;
//   6. interpolate the traces of the updated solution and write them to the
//      other half of the ping-pong trace cache for the next launch.
//
// Global traffic per element-stage is therefore: solution and G read+write,
// metric terms read once, own traces written once, neighbour traces read once
// -- the algorithmic minimum for a stage with one face exchange.
#pragma once

#include <cuda_runtime.h>

#include "physics.cuh"

namespace selfgpu {

constexpr int kMaxP = 8;

enum StageMode { MODE_TRACES = 0, MODE_TENDENCY = 1, MODE_RK = 2 };

struct StageArgs {
  int nEl;
  int mode;
  int flags;  // model-specific presence bits (see the physics policies)
  // geometry (caller owned, FP64)
  const double* __restrict__ dsdx;    // (2,2,P,P,1,nEl)
  const double* __restrict__ J;       // (P,P,1,nEl)
  const double* __restrict__ nHat;    // (2,P,1,4,nEl)
  const double* __restrict__ nScale;  // (P,1,4,nEl)
  const int* __restrict__ sideInfo;   // (5,4,nEl)
  // state (caller owned, FP64)
  double* q;     // (P,P,NV,nEl)
  double* G;     // (P,P,NV,nEl)
  double* dSdt;  // (P,P,NV,nEl), MODE_TENDENCY only
  // engine-owned trace cache, element-blocked: (P, NT, 4, nEl) of the bulk type
  const void* trIn;
  void* trOut;
  // ShallowWater stage-lagged velocity traces (P, 2, 4, nEl)
  const void* velIn;
  void* velOut;
  // model parameters and fields (FP64, caller owned; NULL = absent)
  double g, fC, gamma, Rgas;
  const double* fld[5];
  // RK coefficients: G = a G + dSdt ; q = q + gdt G
  double rk_a, rk_gdt;
  // operator matrices (Lagrange%Init): dgM(ii,i) at [ii + P*i], bM(ii,side), qw
  double dgM[kMaxP * kMaxP];
  double bM[2 * kMaxP];
  double qw[kMaxP];
};

// -------------------------------------------------------------------- models
// Each policy exposes
//   NV  state variables, NT traced fields, NF fields kept per node in smem
//   node(): fill the NF-NV auxiliaries from q (node values)
//   flux(): physical volume flux at a node
//   source(): source term at a node
//   face(): exterior state (exchange done by the kernel, BC here) + Riemann

// LinearShallowWater: q = (u, v, eta); traces (u, v, eta).
// fld[0] = H interior, fld[1] = H boundary, fld[2] = fCori interior.
struct PhysLSW {
  static constexpr int NV = 3, NT = 3, NF = 3;
  static constexpr bool kLaggedVelocity = false;
  template <typename R>
  __device__ static void node(R* /*f*/, const StageArgs&) {}
  template <typename R>
  __device__ static void flux(const R* f, long long gnode, const StageArgs& a, R Fx[3], R Fy[3]) {
    const R H = (R)a.fld[0][gnode];
    const R g = (R)a.g;
    Fx[0] = g * f[2];  // src/models/SELF_LinearShallowWater.f90:470-490
    Fy[0] = (R)0;
    Fx[1] = (R)0;
    Fy[1] = g * f[2];
    Fx[2] = H * f[0];
    Fy[2] = H * f[1];
  }
  template <typename R>
  __device__ static void source(const R* f, long long gnode, int /*t*/, long long /*e*/, int /*PP*/,
                                const StageArgs& a, R S[3]) {
    if (a.fld[2] != nullptr) {  // src/models/SELF_LinearShallowWater.f90:433-439
      const R fc = (R)a.fld[2][gnode];
      S[0] = fc * f[1];
      S[1] = -fc * f[0];
    } else {
      S[0] = (R)0;
      S[1] = (R)0;
    }
    S[2] = (R)0;
  }
  template <typename R>
  __device__ static void face(int bcid, bool physical, const R* L, R* Ext, const R*, const R*, double n1, double n2,
                              double nmag, long long gface, int /*e*/, int /*s*/, int /*i*/, int /*P*/,
                              const StageArgs& a, R out[3]) {
    if (physical) {  // src/models/SELF_LinearShallowWater.f90:323-349
      if (bcid == SG_BC_NONORMALFLOW) {
        reflect<R>(L[0], L[1], n1, n2, Ext[0], Ext[1]);
        Ext[2] = L[2];
      } else {
        Ext[0] = Ext[1] = Ext[2] = (R)0;
      }
    }
    lsw_riemann<R>(L[0], L[1], L[2], Ext[0], Ext[1], Ext[2], (R)a.fld[1][gface], (R)a.g, n1, n2, nmag, out);
  }
};

// ShallowWater: q = (Hu, Hv, H); traces (Hu, Hv, H); aux (u, v).
// fld[0] = topography boundary (radiation exterior H), fld[1] = gradTopography.
struct PhysSW {
  static constexpr int NV = 3, NT = 3, NF = 5;
  static constexpr bool kLaggedVelocity = true;
  template <typename R>
  __device__ static void node(R* f, const StageArgs&) {
    const R H = f[2];  // src/models/SELF_ShallowWater.f90:205-216
    f[3] = f[0] / H;
    f[4] = f[1] / H;
  }
  template <typename R>
  __device__ static void flux(const R* f, long long, const StageArgs& a, R Fx[3], R Fy[3]) {
    sw_flux<R>(f[0], f[1], f[2], f[3], f[4], (R)a.g, Fx, Fy);
  }
  template <typename R>
  __device__ static void source(const R* f, long long gnode, int, long long, int, const StageArgs& a, R S[3]) {
    const R g = (R)a.g, fc = (R)a.fC;  // src/models/SELF_ShallowWater.f90:362-378
    R gx = (R)0, gy = (R)0;
    if (a.fld[1] != nullptr) {
      gx = (R)a.fld[1][2 * gnode];
      gy = (R)a.fld[1][2 * gnode + 1];
    }
    S[0] = -fc * f[1] + g * f[2] * gx;
    S[1] = fc * f[0] + g * f[2] * gy;
    S[2] = (R)0;
  }
  template <typename R>
  __device__ static void face(int bcid, bool physical, const R* L, R* Ext, const R* velL, const R* velR, double n1,
                              double n2, double nmag, long long gface, int, int, int, int, const StageArgs& a,
                              R out[3]) {
    if (physical) {  // src/models/SELF_ShallowWater.f90:305-338
      if (bcid == SG_BC_NONORMALFLOW) {
        reflect<R>(L[0], L[1], n1, n2, Ext[0], Ext[1]);
        Ext[2] = L[2];
      } else {
        Ext[0] = Ext[1] = (R)0;
        Ext[2] = a.fld[0] ? (R)a.fld[0][gface] : (R)0;
      }
    }
    sw_riemann<R>(L[0], L[1], L[2], Ext[0], Ext[1], Ext[2], velL[0], velL[1], velR[0], velR[1], (R)a.g, n1, n2, nmag,
                  out);
  }
};

// CompressibleIdealGas2D: q = (rhoU, rhoV, rho, rhoE); traces
// (rhoU, rhoV, rho, rhoE, u, v, p, rhoH, c) -- the primitive and diagnostic
// traces are interpolated fields, not recomputed from interpolated q.
// fld[0] = environmentalsGradient (2,P,P,2,nEl), fld[1] = environmentals (P,P,2,nEl),
// fld[2..4] = prescribed solution / primitive / diagnostics boundaries (P,4,4,nEl).
struct PhysCIG {
  static constexpr int NV = 4, NT = 9, NF = 9;
  static constexpr bool kLaggedVelocity = false;
  template <typename R>
  __device__ static void node(R* f, const StageArgs& a) {
    R u, v, p, ke, h, c;
    cig_state<R>(f[0], f[1], f[2], f[3], (R)a.gamma, u, v, p, ke, h, c);
    f[4] = u;
    f[5] = v;
    f[6] = p;
    f[7] = h;
    f[8] = c;
  }
  template <typename R>
  __device__ static void flux(const R* f, long long, const StageArgs&, R Fx[4], R Fy[4]) {
    cig_flux<R>(f[0], f[1], f[4], f[5], f[6], f[7], Fx, Fy);
  }
  template <typename R>
  __device__ static void source(const R* f, long long, int t, long long e, int PP, const StageArgs& a, R S[4]) {
    // src/models/SELF_CompressibleIdealGas2D.f90:1339-1360; gravity from
    // variable 1 of environmentalsGradient, drag from variable 2 of environmentals
    R gx = (R)0, gy = (R)0, cd = (R)0;
    if (a.fld[0] != nullptr) {
      const double* gg = a.fld[0] + 2 * (t + (long long)PP * 2 * e);
      gx = (R)gg[0];
      gy = (R)gg[1];
    }
    if (a.fld[1] != nullptr) cd = (R)a.fld[1][t + (long long)PP * (1 + 2 * e)];
    S[0] = -f[2] * gx - cd * f[0];
    S[1] = -f[2] * gy - cd * f[1];
    S[2] = (R)0;
    S[3] = -f[0] * gx - f[0] * gy;
  }
  template <typename R>
  __device__ static void face(int bcid, bool physical, const R* L, R* Ext, const R*, const R*, double n1, double n2,
                              double nmag, long long /*gface*/, int e, int s, int i, int P, const StageArgs& a,
                              R out[4]) {
    if (physical) {  // src/models/SELF_CompressibleIdealGas2D.f90:1256-1317
      if (bcid == SG_BC_NONORMALFLOW) {
        reflect<R>(L[0], L[1], n1, n2, Ext[0], Ext[1]);
        Ext[2] = L[2];
        Ext[3] = L[3];
        reflect<R>(L[4], L[5], n1, n2, Ext[4], Ext[5]);
        Ext[6] = L[6];
        Ext[7] = L[7];
        Ext[8] = L[8];
      } else if ((bcid == SG_BC_PRESCRIBED || bcid == SG_BC_RADIATION) && a.fld[2] != nullptr) {
        const long long b = i + (long long)P * 4 * (s + 4LL * e);  // (i, var, side, el) with 4 vars
        for (int v = 0; v < 4; ++v) Ext[v] = (R)a.fld[2][b + v * P];
        Ext[4] = (R)a.fld[3][b];
        Ext[5] = (R)a.fld[3][b + P];
        Ext[6] = (R)a.fld[3][b + 3 * P];
        Ext[7] = (R)a.fld[4][b + P];
        Ext[8] = (R)a.fld[4][b + 2 * P];
      } else {
        for (int k = 0; k < 9; ++k) Ext[k] = (R)0;
      }
    }
    cig_llf<R>(L, Ext, n1, n2, nmag, out);
  }
};

// ---------------------------------------------------------------- the kernel
// Shared memory per element slot (bulk type R):
//   fld  [NF][P*P]       solution + auxiliaries
//   Fc   [2][NV][P*P]    contravariant flux (reused)
//   own  [4][NT][P]      own traces
//   ext  [4][NT][P]      neighbour traces (flip applied)
//   fb   [4][NV][P]      boundary-normal flux
//   vel  [2][4][2][P]    lagged velocity traces own / neighbour (SW)
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

template <int P, class Phys, typename R, int EPB>
__global__ void __launch_bounds__(EPB* P* P) k_fused_stage(const StageArgs a) {
  constexpr int NV = Phys::NV, NT = Phys::NT, NF = Phys::NF, PP = P * P, N = P - 1;
  using S = Smem<P, Phys, R>;
  __shared__ S sm_all[EPB];
  __shared__ double sdg[PP], sb[2 * P], sqw[P];

  const int tid = threadIdx.x;
  const int slot = tid / PP;
  const int t = tid - slot * PP;  // node index ij = i + P*j
  const int i = t % P, j = t / P;
  S& sm = sm_all[slot];

  for (int k = tid; k < PP; k += blockDim.x) sdg[k] = a.dgM[k];
  for (int k = tid; k < 2 * P; k += blockDim.x) sb[k] = a.bM[k];
  for (int k = tid; k < P; k += blockDim.x) sqw[k] = a.qw[k];

  const long long e = (long long)blockIdx.x * EPB + slot;
  const bool live = e < a.nEl;
  const R* trIn = reinterpret_cast<const R*>(a.trIn);
  R* trOut = reinterpret_cast<R*>(a.trOut);
  const long long gnode = t + (long long)PP * e;

  // ---- 1. solution, auxiliaries
  if (live) {
    R f[NF];
#pragma unroll
    for (int v = 0; v < NV; ++v) f[v] = (R)a.q[t + (long long)PP * (v + NV * e)];
    Phys::template node<R>(f, a);
#pragma unroll
    for (int v = 0; v < NF; ++v) sm.fld[v][t] = f[v];
  }

  if (a.mode != MODE_TRACES) {
    // ---- 1b. contravariant volume flux (registers -> smem)
    if (live) {
      R f[NF];
#pragma unroll
      for (int v = 0; v < NF; ++v) f[v] = sm.fld[v][t];
      R Fx[NV], Fy[NV];
      Phys::template flux<R>(f, gnode, a, Fx, Fy);
      const double2* gp = reinterpret_cast<const double2*>(a.dsdx + 4 * gnode);
      const double2 c1 = gp[0], c2 = gp[1];  // (dsdx11, dsdx21), (dsdx12, dsdx22)
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        sm.Fc[0][v][t] = (R)c1.x * Fx[v] + (R)c1.y * Fy[v];
        sm.Fc[1][v][t] = (R)c2.x * Fx[v] + (R)c2.y * Fy[v];
      }
    }
    // ---- 2a. neighbour traces (and lagged velocities) into smem, flip applied
    if (live) {
      for (int k = t; k < 4 * NT * P; k += PP) {
        const int ii = k % P, fs = k / P, fi = fs % NT, s1 = fs / NT;
        const int* si = a.sideInfo + 5 * (s1 + 4 * e);
        R val = (R)0;
        if (si[4] == 0) {
          const long long e2 = si[2] - 1;
          const int s2 = si[3] / 10 - 1, flip = si[3] % 10;
          const int i2 = flip ? N - ii : ii;
          val = trIn[i2 + P * (fi + NT * (s2 + 4 * e2))];
        }
        sm.ext[s1][fi][ii] = val;
      }
      if constexpr (Phys::kLaggedVelocity) {
        const R* vIn = reinterpret_cast<const R*>(a.velIn);
        for (int k = t; k < 2 * 4 * 2 * P; k += PP) {
          const int ii = k % P, d = (k / P) % 2, s1 = (k / (2 * P)) % 4, which = k / (8 * P);
          R val = (R)0;
          if (which == 0) {
            val = vIn[ii + P * (d + 2 * (s1 + 4 * e))];
          } else {
            const int* si = a.sideInfo + 5 * (s1 + 4 * e);
            if (si[4] == 0) {  // velocity%extBoundary is only ever set by the exchange (H8)
              const long long e2 = si[2] - 1;
              const int s2 = si[3] / 10 - 1, flip = si[3] % 10;
              const int i2 = flip ? N - ii : ii;
              val = vIn[i2 + P * (d + 2 * (s2 + 4 * e2))];
            }
          }
          sm.vel[which][s1][d][ii] = val;
        }
      }
    }
    __syncthreads();
    // ---- 2b. own traces of the current solution (BoundaryInterp)
    if (live) {
      for (int k = t; k < 4 * NT * P; k += PP) {
        const int ii = k % P, fs = k / P, fi = fs % NT, s1 = fs / NT;
        const R* fv = sm.fld[fi];
        R acc = (R)0;
        if (s1 == 0) {
          for (int m = 0; m < P; ++m) acc = acc + (R)sb[m] * fv[ii + P * m];
        } else if (s1 == 1) {
          for (int m = 0; m < P; ++m) acc = acc + (R)sb[m + P] * fv[m + P * ii];
        } else if (s1 == 2) {
          for (int m = 0; m < P; ++m) acc = acc + (R)sb[m + P] * fv[ii + P * m];
        } else {
          for (int m = 0; m < P; ++m) acc = acc + (R)sb[m] * fv[m + P * ii];
        }
        sm.own[s1][fi][ii] = acc;
      }
    }
    __syncthreads();
    // ---- 3. Riemann flux at the 4P face nodes (+ SW velocity cache for the next stage)
    if (live && t < 4 * P) {
      const int s1 = t / P, ii = t % P;
      const int* si = a.sideInfo + 5 * (s1 + 4 * e);
      const int bcid = si[4];
      const bool physical = (bcid != 0) && (si[2] == 0);
      R L[NT], X[NT];
#pragma unroll
      for (int k = 0; k < NT; ++k) {
        L[k] = sm.own[s1][k][ii];
        X[k] = (bcid == 0) ? sm.ext[s1][k][ii] : (R)0;
      }
      const long long gface = ii + (long long)P * (s1 + 4 * e);
      const double2 nh = reinterpret_cast<const double2*>(a.nHat)[gface];
      const double ns = a.nScale[gface];
      R velL[2] = {(R)0, (R)0}, velR[2] = {(R)0, (R)0};
      if constexpr (Phys::kLaggedVelocity) {
        velL[0] = sm.vel[0][s1][0][ii];
        velL[1] = sm.vel[0][s1][1][ii];
        velR[0] = sm.vel[1][s1][0][ii];
        velR[1] = sm.vel[1][s1][1][ii];
        // velocity traces of this stage's solution traces, read by the next stage
        R* vOut = reinterpret_cast<R*>(a.velOut);
        vOut[ii + P * (0 + 2 * (s1 + 4 * e))] = L[0] / L[2];
        vOut[ii + P * (1 + 2 * (s1 + 4 * e))] = L[1] / L[2];
      }
      R out[NV];
      Phys::template face<R>(bcid, physical, L, X, velL, velR, nh.x, nh.y, ns, gface, (int)e, s1, ii, P, a, out);
#pragma unroll
      for (int v = 0; v < NV; ++v) sm.fb[s1][v][ii] = out[v];
    }
    __syncthreads();
    // ---- 4/5. weak divergence + lift, 1/J, dSdt, RK update
    if (live) {
      R f[NF];
#pragma unroll
      for (int v = 0; v < NF; ++v) f[v] = sm.fld[v][t];
      R Src[NV];
      Phys::template source<R>(f, gnode, t, e, PP, a, Src);
      const R Jij = (R)a.J[gnode];
      const R wi = (R)sqw[i], wj = (R)sqw[j];
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        R d = (R)0;
#pragma unroll
        for (int m = 0; m < P; ++m)
          d = d + (R)sdg[m + P * i] * sm.Fc[0][v][m + P * j] + (R)sdg[m + P * j] * sm.Fc[1][v][i + P * m];
        d = d + ((R)sb[i + P] * sm.fb[1][v][j] + (R)sb[i] * sm.fb[3][v][j]) / wi +
            ((R)sb[j + P] * sm.fb[2][v][i] + (R)sb[j] * sm.fb[0][v][i]) / wj;
        const R div = d / Jij;
        const R dsdt = Src[v] - div;
        const long long gi = t + (long long)PP * (v + NV * e);
        if (a.mode == MODE_TENDENCY) {
          a.dSdt[gi] = (double)dsdt;
        } else {
          const double Gn = a.rk_a * a.G[gi] + (double)dsdt;
          a.G[gi] = Gn;
          const double qn = a.q[gi] + a.rk_gdt * Gn;
          a.q[gi] = qn;
          f[v] = (R)qn;
        }
      }
      if (a.mode == MODE_RK) {
        // only this thread reads node t of fld in this phase, so it may overwrite it
        Phys::template node<R>(f, a);
#pragma unroll
        for (int v = 0; v < NF; ++v) sm.fld[v][t] = f[v];
      }
    }
    if (a.mode == MODE_TENDENCY) return;
  }
  __syncthreads();
  // ---- 6. traces of the (updated) solution -> trace cache, element-blocked
  R* o = trOut + (long long)4 * NT * P * e;
  if (live) {
    for (int k = t; k < 4 * NT * P; k += PP) {
      const int ii = k % P, fs = k / P, fi = fs % NT, s1 = fs / NT;
      const R* fv = sm.fld[fi];
      R acc = (R)0;
      if (s1 == 0) {
        for (int m = 0; m < P; ++m) acc = acc + (R)sb[m] * fv[ii + P * m];
      } else if (s1 == 1) {
        for (int m = 0; m < P; ++m) acc = acc + (R)sb[m + P] * fv[m + P * ii];
      } else if (s1 == 2) {
        for (int m = 0; m < P; ++m) acc = acc + (R)sb[m + P] * fv[ii + P * m];
      } else {
        for (int m = 0; m < P; ++m) acc = acc + (R)sb[m] * fv[m + P * ii];
      }
      o[k] = acc;
    }
  }
  if constexpr (Phys::kLaggedVelocity) {
    // Start of a run: the stage-lagged velocity traces equal those of this
    // solution (SetSolution leaves solution%boundary = BoundaryInterp(solution)).
    if (a.mode == MODE_TRACES && a.velOut != nullptr) {
      __syncthreads();
      if (live && t < 4 * P) {
        const int s1 = t / P, ii = t % P;
        R* vOut = reinterpret_cast<R*>(a.velOut);
        const R H = o[ii + P * (2 + NT * s1)];
        vOut[ii + P * (0 + 2 * (s1 + 4 * e))] = o[ii + P * (0 + NT * s1)] / H;
        vOut[ii + P * (1 + 2 * (s1 + 4 * e))] = o[ii + P * (1 + NT * s1)] / H;
      }
    }
  }
}

}  // namespace selfgpu
