// Point-wise physics of the three 2-D models, shared by the drop-in
// per-operator kernels (legacy_ops.cu) and the fused stage kernel
// (fused_stage.cu).  Each function restates one CPU branch of the reference
// with the same left-to-right evaluation order; `R` is the bulk arithmetic
// type (double for the parity form, float for the FP32-bulk form) and normals
// and face scales always arrive in double.
#pragma once

#include <cuda_runtime.h>

// Two builds of the FP64 kernels share these sources.  The default one keeps
// the reference's roundings: it is compiled without multiply-add contraction
// (-fmad=false) and divides where the reference divides (H12: the lift by the
// quadrature weights, 1/J, the density).  A translation unit that defines
// SELFGPU_FP64_PRODUCTION before including the kernel headers builds the
// production FP64 form: compiled with contraction, it multiplies by
// reciprocals instead (FP64 round-off level differences, far inside the 1e-12
// parity bar).  The model policies and the launchers of each build live in
// their own inline namespace, so the two sets of kernel instantiations are
// distinct symbols of one library.
#ifdef SELFGPU_FP64_PRODUCTION
#define SELFGPU_FORM_NS form_production
#define SELFGPU_REF_ROUNDING 0
#else
#define SELFGPU_FORM_NS form_reference
#define SELFGPU_REF_ROUNDING 1
#endif

namespace selfgpu {
inline namespace SELFGPU_FORM_NS {
// true where the bulk type R evaluates with the reference's divisions
template <typename R>
__host__ __device__ constexpr bool ref_rounding() {
  return sizeof(R) == 8 && SELFGPU_REF_ROUNDING;
}
}  // namespace SELFGPU_FORM_NS

#define SG_BC_PRESCRIBED 100
#define SG_BC_RADIATION 101
#define SG_BC_NONORMALFLOW 102

// Reflection of a velocity-like pair across the face normal, used by every
// NONORMALFLOW branch (e.g. src/models/SELF_LinearShallowWater.f90:333-338).
template <typename R>
__device__ __forceinline__ void reflect(R u, R v, double n1, double n2, R& ue, R& ve) {
  const R a = (R)n1, b = (R)n2;
  ue = (b * b - a * a) * u - (R)2 * a * b * v;
  ve = (a * a - b * b) * v - (R)2 * a * b * u;
}

// ------------------------------------------------------------ LinearShallowWater
// Characteristic upwind flux, src/models/SELF_LinearShallowWater.f90:529-551.
template <typename R>
__device__ __forceinline__ void lsw_riemann(R uL, R vL, R etaL, R uR, R vR, R etaR, R Hb, R g, double n1,
                                            double n2, double nmag, R out[3]) {
  const R a = (R)n1, b = (R)n2, s = (R)nmag;
  const R c = sqrt(g * Hb);
  const R unL = uL * a + vL * b;
  const R unR = uR * a + vR * b;
  const R wL = (R)0.5 * (unL / g + etaL / c);
  const R wR = (R)0.5 * (unR / g - etaR / c);
  out[0] = g * c * (wL - wR) * a * s;
  out[1] = g * c * (wL - wR) * b * s;
  out[2] = c * c * (wL + wR) * s;
}

// -------------------------------------------------------------------- ShallowWater
// Local Lax-Friedrichs flux, src/models/SELF_ShallowWater.f90:486-524.
// uvL/uvR are the (stage-lagged) velocity traces.
template <typename R>
__device__ __forceinline__ void sw_riemann(R HuL, R HvL, R HL, R HuR, R HvR, R HR, R uL, R vL, R uR, R vR, R g,
                                           double n1, double n2, double nmag, R out[3]) {
  const R a = (R)n1, b = (R)n2, s = (R)nmag;
  const R unL = uL * a + vL * b;
  const R unR = uR * a + vR * b;
  const R cL = sqrt(g * HL);
  const R cR = sqrt(g * HR);
  const R fL1 = HuL * unL + g * HL * HL * (R)0.5 * a;
  const R fL2 = HvL * unL + g * HL * HL * (R)0.5 * b;
  const R fL3 = HuL * a + HvL * b;
  const R fR1 = HuR * unR + g * HR * HR * (R)0.5 * a;
  const R fR2 = HvR * unR + g * HR * HR * (R)0.5 * b;
  const R fR3 = HuR * a + HvR * b;
  const R alpha = fmax(fmax(fabs(unL + cL), fabs(unR + cR)), fmax(fabs(unL - cL), fabs(unR - cR)));
  out[0] = (R)0.5 * (fL1 + fR1 + alpha * (HuL - HuR)) * s;
  out[1] = (R)0.5 * (fL2 + fR2 + alpha * (HvL - HvR)) * s;
  out[2] = (R)0.5 * (fL3 + fR3 + alpha * (HL - HR)) * s;
}

// Volume flux, src/models/SELF_ShallowWater.f90:400-441.
template <typename R>
__device__ __forceinline__ void sw_flux(R Hu, R Hv, R H, R u, R v, R g, R Fx[3], R Fy[3]) {
  Fx[0] = u * Hu + (R)0.5 * g * H * H;
  Fy[0] = v * Hu;
  Fx[1] = u * Hv;
  Fy[1] = v * Hv + (R)0.5 * g * H * H;
  Fx[2] = Hu;
  Fy[2] = Hv;
}

// --------------------------------------------------------- CompressibleIdealGas2D
// CalculateDiagnostics / ConservativeToPrimitive point values,
// src/models/SELF_CompressibleIdealGas2D.f90:1097-1117, 1149-1163.
// out: u, v, p, rhoKE, rhoH = rhoE + p, c = sqrt(gamma p / rho)
template <typename R>
__device__ __forceinline__ void cig_state(R rhoU, R rhoV, R rho, R rhoE, R gamma, R& u, R& v, R& p, R& rhoKE,
                                          R& rhoH, R& c) {
  if constexpr (!ref_rounding<R>()) {  // FP32 bulk / production FP64: one reciprocal of the density
    const R r = (R)1 / rho;
    u = rhoU * r;
    v = rhoV * r;
    rhoKE = (R)0.5 * (rhoU * u + rhoV * v);
    p = (gamma - (R)1) * (rhoE - rhoKE);
    rhoH = rhoE + p;
    c = sqrt(gamma * p * r);
  } else {  // the reference's divisions
    u = rhoU / rho;
    v = rhoV / rho;
    rhoKE = (R)0.5 * (rhoU * u + rhoV * v);
    p = (gamma - (R)1) * (rhoE - rhoKE);
    rhoH = rhoE + p;
    c = sqrt(gamma * p / rho);
  }
}

// NaiveLLF, src/models/SELF_CompressibleIdealGas2D.f90:1486-1534.
// L/R hold (rhoU, rhoV, rho, rhoE, u, v, p, rhoH, c).
template <typename R>
__device__ __forceinline__ void cig_llf(const R L[9], const R Rt[9], double n1, double n2, double nmag, R out[4]) {
  const R a = (R)n1, b = (R)n2, s = (R)nmag;
  const R unL = L[4] * a + L[5] * b;
  const R unR = Rt[4] * a + Rt[5] * b;
  R fL[4], fR[4];
  fL[0] = unL * L[0] + L[6] * a;
  fL[1] = unL * L[1] + L[6] * b;
  fL[2] = L[0] * a + L[1] * b;
  fL[3] = unL * L[7];
  fR[0] = unR * Rt[0] + Rt[6] * a;
  fR[1] = unR * Rt[1] + Rt[6] * b;
  fR[2] = Rt[0] * a + Rt[1] * b;
  fR[3] = unR * Rt[7];
  const R alpha = fmax(fabs(unL), fabs(unR)) + fmax(fabs(L[8]), fabs(Rt[8]));
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = (R)0.5 * (fL[k] + fR[k] + alpha * (L[k] - Rt[k])) * s;
}

// Volume flux, src/models/SELF_CompressibleIdealGas2D.f90:1384-1432.
template <typename R>
__device__ __forceinline__ void cig_flux(R rhoU, R rhoV, R u, R v, R p, R rhoH, R Fx[4], R Fy[4]) {
  Fx[0] = u * rhoU + p;
  Fy[0] = v * rhoU;
  Fx[1] = u * rhoV;
  Fy[1] = v * rhoV + p;
  Fx[2] = rhoU;
  Fy[2] = rhoV;
  Fx[3] = u * rhoH;
  Fy[3] = v * rhoH;
}

}  // namespace selfgpu
