// Drop-in replacements for SELF's per-operator HIP wrappers (FP64).
//
// Same symbol names and arguments as the reference (see include/selfgpu.h for
// the file:line each replaces); each wrapper dereferences the real** it gets,
// launches on the legacy default stream and returns without synchronising, as
// the reference does.  Unlike the reference kernels (one block per
// (var, element), one thread per node, strided uncoalesced traces), these are
// flat grid-stride kernels over contiguous outputs so that every warp reads and
// writes consecutive addresses; the arithmetic of each output follows the CPU
// branch of the reference term by term.  The whole-stage fused kernels in
// fused_stage.cu are the fast path; these exist so an unmodified SELF caller
// can use the library operator by operator.
#include <cuda_runtime.h>

#include <string>

#include "physics.cuh"
#include "selfgpu_internal.h"

namespace selfgpu {
namespace {

constexpr int kThreads = 256;

inline int blocks_for(long long n) {
  long long b = (n + kThreads - 1) / kThreads;
  if (b < 1) b = 1;
  if (b > 148LL * 64) b = 148LL * 64;  // grid-stride beyond 64 CTAs per SM
  return (int)b;
}

inline void check_launch(const char* name) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) set_error(SELFGPU_ERR_CUDA, std::string(name) + ": " + cudaGetErrorString(e));
}

#define GRID_STRIDE(k, n) for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < (n); \
                               k += (long long)gridDim.x * blockDim.x)

// ------------------------------------------------------------------ Lagrange
// src/SELF_Lagrange.f90:741-789; iM(ii,m) at iM[ii + P*m]
__global__ void k_scalar_grid_interp(const double* __restrict__ iM, const double* __restrict__ f,
                                     double* __restrict__ fo, int N, int M, long long n) {
  const int P = N + 1, Q = M + 1;
  GRID_STRIDE(k, n) {
    const int i = k % Q, j = (k / Q) % Q;
    const long long ve = k / ((long long)Q * Q);
    const double* fe = f + ve * P * P;
    double fij = 0.0;
    for (int jj = 0; jj < P; ++jj) {
      double fi = 0.0;
      for (int ii = 0; ii < P; ++ii) fi = fi + fe[ii + P * jj] * iM[ii + P * i];
      fij = fij + fi * iM[jj + P * j];
    }
    fo[k] = fij;
  }
}

// src/SELF_Lagrange.f90:824-875
__global__ void k_vector_grid_interp(const double* __restrict__ iM, const double* __restrict__ f,
                                     double* __restrict__ fo, int N, int M, long long n) {
  const int P = N + 1, Q = M + 1;
  GRID_STRIDE(k, n) {  // k enumerates (dir, i, j, var*el)
    const int d = k & 1;
    const long long kn = k >> 1;
    const int i = kn % Q, j = (kn / Q) % Q;
    const long long ve = kn / ((long long)Q * Q);
    const double* fe = f + ve * 2 * P * P;
    double o = 0.0;
    for (int jj = 0; jj < P; ++jj) {
      double fi = 0.0;
      for (int ii = 0; ii < P; ++ii) fi = fi + fe[d + 2 * (ii + P * jj)] * iM[ii + P * i];
      o = o + fi * iM[jj + P * j];
    }
    fo[k] = o;
  }
}

// src/SELF_Lagrange.f90:2241-2270; one thread per (i, var, el) writes 4 sides
__global__ void k_scalar_boundary_interp(const double* __restrict__ bM, const double* __restrict__ f,
                                         double* __restrict__ fb, int N, int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P;
    const long long ve = k / P;
    const int v = ve % nVar;
    const long long e = ve / nVar;
    const double* fe = f + ve * P * P;
    double b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    for (int ii = 0; ii < P; ++ii) {
      b1 = b1 + bM[ii] * fe[i + P * ii];
      b2 = b2 + bM[ii + P] * fe[ii + P * i];
      b3 = b3 + bM[ii + P] * fe[i + P * ii];
      b4 = b4 + bM[ii] * fe[ii + P * i];
    }
    double* o = fb + i + (long long)P * (v + (long long)nVar * 4 * e);
    const long long ss = (long long)P * nVar;
    o[0] = b1;
    o[ss] = b2;
    o[2 * ss] = b3;
    o[3 * ss] = b4;
  }
}

// src/SELF_Lagrange.f90:2284-2316 (C = 2) and 2330-2366 (C = 4): components fastest
template <int C>
__global__ void k_multi_boundary_interp(const double* __restrict__ bM, const double* __restrict__ f,
                                        double* __restrict__ fb, int N, int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {  // k enumerates (comp, i, var, el)
    const int c = k % C;
    const int i = (k / C) % P;
    const long long ve = k / ((long long)C * P);
    const int v = ve % nVar;
    const long long e = ve / nVar;
    const double* fe = f + ve * C * P * P;
    double b1 = 0, b2 = 0, b3 = 0, b4 = 0;
    for (int ii = 0; ii < P; ++ii) {
      b1 = b1 + bM[ii] * fe[c + C * (i + P * ii)];
      b2 = b2 + bM[ii + P] * fe[c + C * (ii + P * i)];
      b3 = b3 + bM[ii + P] * fe[c + C * (i + P * ii)];
      b4 = b4 + bM[ii] * fe[c + C * (ii + P * i)];
    }
    double* o = fb + c + C * (i + (long long)P * (v + (long long)nVar * 4 * e));
    const long long ss = (long long)C * P * nVar;
    o[0] = b1;
    o[ss] = b2;
    o[2 * ss] = b3;
    o[3 * ss] = b4;
  }
}

// src/SELF_Lagrange.f90:1424-1463
__global__ void k_vector_gradient(const double* __restrict__ dM, const double* __restrict__ f,
                                  double* __restrict__ gf, int N, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {  // k enumerates (i, j, var*el)
    const int i = k % P, j = (k / P) % P;
    const long long ve = k / ((long long)P * P);
    const double* fe = f + ve * 2 * P * P;
    double g11 = 0, g21 = 0, g12 = 0, g22 = 0;
    for (int ii = 0; ii < P; ++ii) {
      g11 = g11 + dM[ii + P * i] * fe[0 + 2 * (ii + P * j)];
      g21 = g21 + dM[ii + P * i] * fe[1 + 2 * (ii + P * j)];
      g12 = g12 + dM[ii + P * j] * fe[0 + 2 * (i + P * ii)];
      g22 = g22 + dM[ii + P * j] * fe[1 + 2 * (i + P * ii)];
    }
    double* o = gf + 4 * k;
    o[0] = g11;
    o[1] = g21;
    o[2] = g12;
    o[3] = g22;
  }
}

// src/SELF_Lagrange.f90:1589-1625
__global__ void k_vector_dg_divergence(const double* __restrict__ dgM, const double* __restrict__ bM,
                                       const double* __restrict__ qw, const double* __restrict__ f,
                                       const double* __restrict__ bf, double* __restrict__ df, int N, int nVar,
                                       long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P, j = (k / P) % P;
    const long long ve = k / ((long long)P * P);
    const int v = ve % nVar;
    const long long e = ve / nVar;
    const double* fe = f + ve * 2 * P * P;
    double d = 0.0;
    for (int ii = 0; ii < P; ++ii)
      d = d + dgM[ii + P * i] * fe[0 + 2 * (ii + P * j)] + dgM[ii + P * j] * fe[1 + 2 * (i + P * ii)];
    const double* b = bf + (long long)P * (v + (long long)nVar * 4 * e);
    const long long ss = (long long)P * nVar;
    d = d + (bM[i + P] * b[j + ss] + bM[i] * b[j + 3 * ss]) / qw[i] +
        (bM[j + P] * b[i + 2 * ss] + bM[j] * b[i]) / qw[j];
    df[k] = d;
  }
}

// src/SELF_Data.f90:1570-1607
__global__ void k_determinant(const double* __restrict__ t, double* __restrict__ det, long long n) {
  GRID_STRIDE(k, n) {
    const double* a = t + 4 * k;
    det[k] = a[0] * a[3] - a[2] * a[1];
  }
}

// src/SELF_Geometry.f90:448-457 (dsdx(:,1) = (dy/ds2, -dx/ds2), dsdx(:,2) = (-dy/ds1, dx/ds1))
__global__ void k_contravariant_basis(const double* __restrict__ dxds, double* __restrict__ dsdx, long long n) {
  GRID_STRIDE(k, n) {
    const double* a = dxds + 4 * k;
    double* o = dsdx + 4 * k;
    o[0] = a[3];
    o[1] = -a[2];
    o[2] = -a[1];
    o[3] = a[0];
  }
}

// Sign adjustment of dsdx on the faces: outward on East/North for J > 0,
// src/SELF_Geometry.f90:462-520 (fac), applied to all four components.
__global__ void k_adjust_boundary_basis(double* __restrict__ dsdxB, const double* __restrict__ JB, int N,
                                        long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {  // k enumerates (i, side, el) of the scalar face layout
    const int s = (k / P) % 4;
    const double j = JB[k];
    const double fac = (s == 1 || s == 2) ? copysign(1.0, j) : -copysign(1.0, j);
    double* o = dsdxB + 4 * k;
    for (int q = 0; q < 4; ++q) o[q] = o[q] * fac;
  }
}

// nHat and nScale from the (unsigned) face contravariant basis, then the sign
// adjustment, as CalculateContravariantBasis_SEMQuad does on the host
// (src/SELF_Geometry.f90:458-522).
__global__ void k_face_normals(double* __restrict__ dsdxB, const double* __restrict__ JB, double* __restrict__ nHat,
                               double* __restrict__ nScale, int N, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int s = (k / P) % 4;
    const double j = JB[k];
    const double fac = (s == 1 || s == 2) ? copysign(1.0, j) : -copysign(1.0, j);
    double* t = dsdxB + 4 * k;
    const int col = (s == 0 || s == 2) ? 1 : 0;
    const double a0 = t[2 * col], a1 = t[2 * col + 1];
    const double mag = sqrt(a0 * a0 + a1 * a1);
    nScale[k] = mag;
    nHat[2 * k] = fac * a0 / mag;
    nHat[2 * k + 1] = fac * a1 / mag;
    for (int q = 0; q < 4; ++q) t[q] = t[q] * fac;
  }
}

// ---------------------------------------------------------------- MappedData
// src/SELF_MappedData.f90:955-1078 (BR1 gradient, weak form)
__global__ void k_gradient_br(const double* __restrict__ f, const double* __restrict__ avgB,
                              const double* __restrict__ dsdx, const double* __restrict__ J,
                              const double* __restrict__ nHat, const double* __restrict__ nScale,
                              double* __restrict__ gradF, const double* __restrict__ dgM,
                              const double* __restrict__ bM, const double* __restrict__ qw, int N, int nVar,
                              long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P, j = (k / P) % P;
    const long long ve = k / ((long long)P * P);
    const int v = ve % nVar;
    const long long e = ve / nVar;
    const double* fe = f + ve * P * P;
    const double* ge = dsdx + e * 4 * P * P;
    double gx = 0.0, gy = 0.0;
    for (int ii = 0; ii < P; ++ii) {
      const double* a = ge + 4 * (ii + P * j);
      const double* b = ge + 4 * (i + P * ii);
      double f1 = fe[ii + P * j] * a[0];
      double f2 = fe[i + P * ii] * b[2];
      gx = gx + dgM[ii + P * i] * f1 + dgM[ii + P * j] * f2;
      f1 = fe[ii + P * j] * a[1];
      f2 = fe[i + P * ii] * b[3];
      gy = gy + dgM[ii + P * i] * f1 + dgM[ii + P * j] * f2;
    }
    const double* av = avgB + (long long)P * (v + (long long)nVar * 4 * e);
    const long long ss = (long long)P * nVar;
    const double* nh = nHat + 2 * P * 4 * e;
    const double* ns = nScale + P * 4 * e;
    auto NH = [&](int d, int q, int s) { return nh[d + 2 * (q + P * s)]; };
    auto NS = [&](int q, int s) { return ns[q + P * s]; };
    double f1 = av[j + ss] * NH(0, j, 1) * NS(j, 1);
    double f2 = av[j + 3 * ss] * NH(0, j, 3) * NS(j, 3);
    gx = gx + (f1 * bM[i + P] + f2 * bM[i]) / qw[i];
    f1 = av[i + 2 * ss] * NH(0, i, 2) * NS(i, 2);
    f2 = av[i] * NH(0, i, 0) * NS(i, 0);
    gx = gx + (f1 * bM[j + P] + f2 * bM[j]) / qw[j];
    f1 = av[j + ss] * NH(1, j, 1) * NS(j, 1);
    f2 = av[j + 3 * ss] * NH(1, j, 3) * NS(j, 3);
    gy = gy + (f1 * bM[i + P] + f2 * bM[i]) / qw[i];
    f1 = av[i + 2 * ss] * NH(1, i, 2) * NS(i, 2);
    f2 = av[i] * NH(1, i, 0) * NS(i, 0);
    gy = gy + (f1 * bM[j + P] + f2 * bM[j]) / qw[j];
    const double Jij = J[i + P * (j + P * e)];
    gradF[2 * k] = gx / Jij;
    gradF[2 * k + 1] = gy / Jij;
  }
}

// src/SELF_MappedData.f90:1080-1149 (strong form)
__global__ void k_gradient_sf(const double* __restrict__ f, const double* __restrict__ dsdx,
                              const double* __restrict__ J, double* __restrict__ gradF, const double* __restrict__ dM,
                              int N, int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P, j = (k / P) % P;
    const long long ve = k / ((long long)P * P);
    const long long e = ve / nVar;
    const double* fe = f + ve * P * P;
    const double* ge = dsdx + e * 4 * P * P;
    double gx = 0.0, gy = 0.0;
    for (int ii = 0; ii < P; ++ii) {
      const double* a = ge + 4 * (ii + P * j);
      const double* b = ge + 4 * (i + P * ii);
      double f1 = fe[ii + P * j] * a[0];
      double f2 = fe[i + P * ii] * b[2];
      gx = gx + dM[ii + P * i] * f1 + dM[ii + P * j] * f2;
      f1 = fe[ii + P * j] * a[1];
      f2 = fe[i + P * ii] * b[3];
      gy = gy + dM[ii + P * i] * f1 + dM[ii + P * j] * f2;
    }
    const double Jij = J[i + P * (j + P * e)];
    gradF[2 * k] = gx / Jij;
    gradF[2 * k + 1] = gy / Jij;
  }
}

// src/SELF_MappedData.f90:1235-1268 (C = 1) and the vector analogue (C = 2)
template <int C>
__global__ void k_jacobian_weight(double* __restrict__ f, const double* __restrict__ J, int N, int nVar,
                                  long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const long long node = k / C;
    const int ij = node % (P * P);
    const long long e = node / ((long long)P * P * nVar);
    f[k] = f[k] / J[ij + (long long)P * P * e];
  }
}

// src/SELF_MappedData.f90:2220-2269
__global__ void k_contravariant_projection(double* __restrict__ f, const double* __restrict__ dsdx, int N, int nVar,
                                           long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int ij = k % (P * P);
    const long long e = k / ((long long)P * P * nVar);
    const double* g = dsdx + 4 * (ij + (long long)P * P * e);
    const double Fx = f[2 * k], Fy = f[2 * k + 1];
    f[2 * k] = g[0] * Fx + g[1] * Fy;
    f[2 * k + 1] = g[2] * Fx + g[3] * Fy;
  }
}

// src/SELF_MappedData.f90:834-917 (C = 1) and 1870-1958 (C = 2): one thread per
// (component, node, var, side, element) output of extBoundary.
template <int C>
__global__ void k_side_exchange(double* __restrict__ ext, const double* __restrict__ bnd,
                                const int* __restrict__ sideInfo, const int* __restrict__ elemToRank, int rankId,
                                int offset, int N, int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int c = k % C;
    const int i1 = (k / C) % P;
    const long long r = k / ((long long)C * P);  // (var, side, el)
    const int v = r % nVar;
    const int s1 = (r / nVar) % 4;
    const long long e1 = r / (4LL * nVar);
    const int* si = sideInfo + 5 * (s1 + 4 * e1);
    const int bcid = si[4];
    if (bcid != 0) continue;
    const int e2g = si[2];
    if (elemToRank != nullptr && elemToRank[e2g - 1] != rankId) continue;
    const int s2 = si[3] / 10, flip = si[3] - s2 * 10;
    const long long e2 = (long long)e2g - 1 - offset;
    const long long nEl = n / (4LL * C * P * nVar);
    if (e2 < 0 || e2 >= nEl || s2 < 1 || s2 > 4) continue;  // malformed record: leave ext untouched
    int i2;
    if (flip == 0) i2 = i1;
    else if (flip == 1) i2 = N - i1;
    else continue;
    ext[k] = bnd[c + C * (i2 + (long long)P * (v + (long long)nVar * ((s2 - 1) + 4 * e2)))];
  }
}

// src/SELF_MappedData.f90:919-953
__global__ void k_bassi_rebay(double* __restrict__ avg, const double* __restrict__ bnd,
                              const double* __restrict__ ext, long long n) {
  GRID_STRIDE(k, n) avg[k] = 0.5 * (bnd[k] + ext[k]);
}

// ------------------------------------------------------------------- Model2D
// src/SELF_Model2D.f90:734-748 (workSol may have nWork != nVar variables)
__global__ void k_update_grk(double* __restrict__ grk, double* __restrict__ sol, const double* __restrict__ dSdt,
                             double a, double g, double dt, int nWork, int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long ve = k / P2;
    const int v = ve % nVar;
    const long long e = ve / nVar;
    const long long kw = ij + (long long)P2 * (v + (long long)nWork * e);
    const double G = a * grk[kw] + dSdt[k];
    grk[kw] = G;
    sol[k] = sol[k] + g * dt * G;
  }
}

__global__ void k_update_solution(double* __restrict__ sol, const double* __restrict__ dSdt, double dt, long long n) {
  GRID_STRIDE(k, n) sol[k] = sol[k] + dt * dSdt[k];
}

// src/SELF_Model2D.f90:845-857
__global__ void k_dsdt(const double* __restrict__ div, const double* __restrict__ src, double* __restrict__ dSdt,
                       long long n) {
  GRID_STRIDE(k, n) dSdt[k] = src[k] - div[k];
}

// -------------------------------------------------------- LinearShallowWater
// src/models/SELF_LinearShallowWater.f90:298-355; thread per (i, side, el)
__global__ void k_lsw_bc(const double* __restrict__ sol, double* __restrict__ ext, const double* __restrict__ nHat,
                         const int* __restrict__ sideInfo, int N, int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P, s = (k / P) % 4;
    const long long e = k / (4LL * P);
    const int* si = sideInfo + 5 * (s + 4 * e);
    if (si[2] != 0) continue;
    const long long ss = P;  // stride between variables in the face layout
    const long long base = i + (long long)P * nVar * (s + 4 * e);
    if (si[4] == SG_BC_NONORMALFLOW) {
      double ue, ve;
      reflect<double>(sol[base], sol[base + ss], nHat[2 * k], nHat[2 * k + 1], ue, ve);
      ext[base] = ue;
      ext[base + ss] = ve;
      ext[base + 2 * ss] = sol[base + 2 * ss];
    } else {
      ext[base] = 0.0;
      ext[base + ss] = 0.0;
      ext[base + 2 * ss] = 0.0;
    }
  }
}

__global__ void k_lsw_source(double* __restrict__ src, const double* __restrict__ sol, const double* __restrict__ f,
                             int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {  // (ij, el)
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    const double fc = f[k];
    src[b] = fc * sol[b + P2];
    src[b + P2] = -fc * sol[b];
    src[b + 2 * P2] = 0.0;
  }
}

__global__ void k_lsw_flux(double* __restrict__ flux, const double* __restrict__ sol, const double* __restrict__ H,
                           double g, int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    const double Hh = H[k];
    flux[2 * b] = g * sol[b + 2 * P2];
    flux[2 * b + 1] = 0.0;
    flux[2 * (b + P2)] = 0.0;
    flux[2 * (b + P2) + 1] = g * sol[b + 2 * P2];
    flux[2 * (b + 2 * P2)] = Hh * sol[b];
    flux[2 * (b + 2 * P2) + 1] = Hh * sol[b + P2];
  }
}

__global__ void k_lsw_riemann(double* __restrict__ flux, const double* __restrict__ sol,
                              const double* __restrict__ ext, const double* __restrict__ H,
                              const double* __restrict__ nHat, const double* __restrict__ nScale, double g, int N,
                              int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {  // (i, side, el)
    const int i = k % P;
    const long long se = k / P;
    const long long base = i + (long long)P * nVar * se;
    double out[3];
    lsw_riemann<double>(sol[base], sol[base + P], sol[base + 2 * P], ext[base], ext[base + P], ext[base + 2 * P],
                        H[k], g, nHat[2 * k], nHat[2 * k + 1], nScale[k], out);
    flux[base] = out[0];
    flux[base + P] = out[1];
    flux[base + 2 * P] = out[2];
  }
}

// -------------------------------------------------------------- ShallowWater
__global__ void k_sw_bc(const double* __restrict__ sol, double* __restrict__ ext, const double* __restrict__ topoB,
                        const double* __restrict__ nHat, const int* __restrict__ sideInfo, int N, int nVar,
                        long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P, s = (k / P) % 4;
    const long long e = k / (4LL * P);
    const int* si = sideInfo + 5 * (s + 4 * e);
    if (si[2] != 0) continue;
    const long long base = i + (long long)P * nVar * (s + 4 * e);
    if (si[4] == SG_BC_NONORMALFLOW) {
      double ue, ve;
      reflect<double>(sol[base], sol[base + P], nHat[2 * k], nHat[2 * k + 1], ue, ve);
      ext[base] = ue;
      ext[base + P] = ve;
      ext[base + 2 * P] = sol[base + 2 * P];
    } else {
      ext[base] = 0.0;
      ext[base + P] = 0.0;
      ext[base + 2 * P] = topoB[k];
    }
  }
}

__global__ void k_sw_source(double* __restrict__ src, const double* __restrict__ sol, const double* __restrict__ gH,
                            double fC, double g, int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    src[b] = -fC * sol[b + P2] + g * sol[b + 2 * P2] * gH[2 * k];
    src[b + P2] = fC * sol[b] + g * sol[b + 2 * P2] * gH[2 * k + 1];
    src[b + 2 * P2] = 0.0;
  }
}

__global__ void k_sw_flux(double* __restrict__ flux, const double* __restrict__ sol, const double* __restrict__ vel,
                          double g, int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    double Fx[3], Fy[3];
    sw_flux<double>(sol[b], sol[b + P2], sol[b + 2 * P2], vel[2 * k], vel[2 * k + 1], g, Fx, Fy);
    for (int v = 0; v < 3; ++v) {
      flux[2 * (b + v * P2)] = Fx[v];
      flux[2 * (b + v * P2) + 1] = Fy[v];
    }
  }
}

__global__ void k_sw_riemann(double* __restrict__ flux, const double* __restrict__ sol, const double* __restrict__ ext,
                             const double* __restrict__ vel, const double* __restrict__ velExt,
                             const double* __restrict__ nHat, const double* __restrict__ nScale, double g, int N,
                             int nVar, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P;
    const long long se = k / P;
    const long long base = i + (long long)P * nVar * se;
    double out[3];
    sw_riemann<double>(sol[base], sol[base + P], sol[base + 2 * P], ext[base], ext[base + P], ext[base + 2 * P],
                       vel[2 * k], vel[2 * k + 1], velExt[2 * k], velExt[2 * k + 1], g, nHat[2 * k],
                       nHat[2 * k + 1], nScale[k], out);
    flux[base] = out[0];
    flux[base + P] = out[1];
    flux[base + 2 * P] = out[2];
  }
}

// velocity = (Hu, Hv)/H on interior nodes (first kernel) and on face nodes
// (second), src/models/SELF_ShallowWater.f90:205-236
__global__ void k_sw_velocity(const double* __restrict__ sol, double* __restrict__ vel, int stride, int nVar,
                              long long n) {
  GRID_STRIDE(k, n) {  // k enumerates (node-or-face-node, block)
    const int q = k % stride;
    const long long blk = k / stride;
    const long long b = q + (long long)stride * nVar * blk;
    const double H = sol[b + 2 * stride];
    vel[2 * k] = sol[b] / H;
    vel[2 * k + 1] = sol[b + stride] / H;
  }
}

// ---------------------------------------------------- CompressibleIdealGas2D
__global__ void k_cig_source(double* __restrict__ src, const double* __restrict__ sol,
                             const double* __restrict__ envGrad, int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    const double* gg = envGrad + 2 * (ij + (long long)P2 * 2 * e);  // variable 1 of 2
    const double gx = gg[0], gy = gg[1];
    const double rhou = sol[b], rhov = sol[b + P2], rho = sol[b + 2 * P2];
    src[b] = -rho * gx;
    src[b + P2] = -rho * gy;
    src[b + 2 * P2] = 0.0;
    src[b + 3 * P2] = -rhou * gx - rhou * gy;
    (void)rhov;
  }
}

__global__ void k_cig_flux(double* __restrict__ flux, const double* __restrict__ sol, const double* __restrict__ prim,
                           const double* __restrict__ diag, int N, int nVar, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    double Fx[4], Fy[4];
    // rhoH = rhoE + p, the CPU diagnostic (SELF_CompressibleIdealGas2D.f90:1110)
    const double rhoH = diag ? diag[b + P2] : sol[b + 3 * P2] + prim[b + 3 * P2];
    cig_flux<double>(sol[b], sol[b + P2], prim[b], prim[b + P2], prim[b + 3 * P2], rhoH, Fx, Fy);
    for (int v = 0; v < 4; ++v) {
      flux[2 * (b + v * P2)] = Fx[v];
      flux[2 * (b + v * P2) + 1] = Fy[v];
    }
  }
}

__global__ void k_cig_llf(double* __restrict__ flux, const double* __restrict__ sol, const double* __restrict__ solE,
                          const double* __restrict__ prim, const double* __restrict__ primE,
                          const double* __restrict__ diag, const double* __restrict__ diagE,
                          const double* __restrict__ nHat, const double* __restrict__ nScale, int N, int nVar,
                          int nDiag, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P;
    const long long se = k / P;
    const long long b = i + (long long)P * nVar * se;
    const long long bd = i + (long long)P * nDiag * se;
    double L[9], R[9], out[4];
    for (int v = 0; v < 4; ++v) {
      L[v] = sol[b + v * P];
      R[v] = solE[b + v * P];
    }
    L[4] = prim[b];
    L[5] = prim[b + P];
    L[6] = prim[b + 3 * P];
    R[4] = primE[b];
    R[5] = primE[b + P];
    R[6] = primE[b + 3 * P];
    L[7] = diag[bd + P];
    L[8] = diag[bd + 2 * P];
    R[7] = diagE[bd + P];
    R[8] = diagE[bd + 2 * P];
    cig_llf<double>(L, R, nHat[2 * k], nHat[2 * k + 1], nScale[k], out);
    for (int v = 0; v < 4; ++v) flux[b + v * P] = out[v];
  }
}

__global__ void k_cig_bc(const double* __restrict__ in, double* __restrict__ ext, const double* __restrict__ presc,
                         const double* __restrict__ nHat, const int* __restrict__ sideInfo, int N, int nv,
                         int reflectPair, long long n) {
  const int P = N + 1;
  GRID_STRIDE(k, n) {
    const int i = k % P, s = (k / P) % 4;
    const long long e = k / (4LL * P);
    const int* si = sideInfo + 5 * (s + 4 * e);
    if (si[2] != 0) continue;
    const long long base = i + (long long)P * nv * (s + 4 * e);
    if (si[4] == SG_BC_NONORMALFLOW) {
      for (int v = 0; v < nv; ++v) ext[base + v * P] = in[base + v * P];
      if (reflectPair) {
        double ue, ve;
        reflect<double>(in[base], in[base + P], nHat[2 * k], nHat[2 * k + 1], ue, ve);
        ext[base] = ue;
        ext[base + P] = ve;
      }
    } else if (si[4] == SG_BC_PRESCRIBED || si[4] == SG_BC_RADIATION) {
      for (int v = 0; v < nv; ++v) ext[base + v * P] = presc[base + v * P];
    }
  }
}

// CalculateDiagnostics (mode 0), ConservativeToPrimitive (mode 1),
// ConservativeToEntropy (mode 2); src/models/SELF_CompressibleIdealGas2D.f90:1076-1215
__global__ void k_cig_pointwise(const double* __restrict__ sol, double* __restrict__ out, double gamma, double Rg,
                                int mode, int N, int nVar, int nOut, long long n) {
  const int P2 = (N + 1) * (N + 1);
  GRID_STRIDE(k, n) {
    const int ij = k % P2;
    const long long e = k / P2;
    const long long b = ij + (long long)P2 * nVar * e;
    const long long o = ij + (long long)P2 * nOut * e;
    const double rhoU = sol[b], rhoV = sol[b + P2], rho = sol[b + 2 * P2], rhoE = sol[b + 3 * P2];
    double u, v, p, rhoKE, rhoH, c;
    cig_state<double>(rhoU, rhoV, rho, rhoE, gamma, u, v, p, rhoKE, rhoH, c);
    if (mode == 0) {
      out[o] = rhoKE;
      out[o + P2] = rhoH;
      out[o + 2 * P2] = c;
      out[o + 3 * P2] = (2.0 / 3.0) * ((rhoE - rhoKE) / rho) / Rg;
    } else if (mode == 1) {
      out[o] = u;
      out[o + P2] = v;
      out[o + 2 * P2] = rho;
      out[o + 3 * P2] = p;
    } else {
      const double s = log(p) - gamma * log(rho);
      out[o] = u * rho / p;
      out[o + P2] = v * rho / p;
      out[o + 2 * P2] = (gamma - s) / (gamma - 1.0) - rhoKE / p;
      out[o + 3 * P2] = -rho / p;
    }
  }
}

}  // namespace
}  // namespace selfgpu

using namespace selfgpu;

#define LAUNCH(kernel, n, ...)                                   \
  do {                                                           \
    long long n_ = (n);                                          \
    if (n_ > 0) kernel<<<blocks_for(n_), kThreads>>>(__VA_ARGS__, n_); \
    check_launch(#kernel);                                       \
  } while (0)

extern "C" {

void ScalarGridInterp_2D_gpu_wrapper(double** iMatrix, double** f, double** fInterp, int N, int M, int nVar, int nEl) {
  LAUNCH(k_scalar_grid_interp, (long long)(M + 1) * (M + 1) * nVar * nEl, *iMatrix, *f, *fInterp, N, M);
}
void VectorGridInterp_2D_gpu_wrapper(double** iMatrix, double** f, double** fInterp, int N, int M, int nVar, int nEl) {
  LAUNCH(k_vector_grid_interp, 2LL * (M + 1) * (M + 1) * nVar * nEl, *iMatrix, *f, *fInterp, N, M);
}
void ScalarBoundaryInterp_2D_gpu_wrapper(double** bMatrix, double** f, double** fBound, int N, int nVar, int nEl) {
  LAUNCH(k_scalar_boundary_interp, (long long)(N + 1) * nVar * nEl, *bMatrix, *f, *fBound, N, nVar);
}
void VectorBoundaryInterp_2D_gpu_wrapper(double** bMatrix, double** f, double** fBound, int N, int nVar, int nEl) {
  LAUNCH(k_multi_boundary_interp<2>, 2LL * (N + 1) * nVar * nEl, *bMatrix, *f, *fBound, N, nVar);
}
void TensorBoundaryInterp_2D_gpu_wrapper(double** bMatrix, double** f, double** fBound, int N, int nVar, int nEl) {
  LAUNCH(k_multi_boundary_interp<4>, 4LL * (N + 1) * nVar * nEl, *bMatrix, *f, *fBound, N, nVar);
}
void VectorGradient_2D_gpu_wrapper(double** dMatrix, double** f, double** df, int N, int nVar, int nEl) {
  LAUNCH(k_vector_gradient, (long long)(N + 1) * (N + 1) * nVar * nEl, *dMatrix, *f, *df, N);
}
void VectorDGDivergence_2D_gpu_wrapper(double** dgMatrix, double** bMatrix, double** qWeights, double** f, double** bf,
                                       double** df, int N, int nVar, int nEl) {
  LAUNCH(k_vector_dg_divergence, (long long)(N + 1) * (N + 1) * nVar * nEl, *dgMatrix, *bMatrix, *qWeights, *f, *bf,
         *df, N, nVar);
}
void Determinant_Tensor2D_gpu_wrapper(double** tensor, double** detTensor, int N, int nVar, int nEl) {
  LAUNCH(k_determinant, (long long)(N + 1) * (N + 1) * nVar * nEl, *tensor, *detTensor);
}
void CalculateContravariantBasis_SEMQuad_gpu_wrapper(double** dxds, double** dsdx, int N, int nEl) {
  LAUNCH(k_contravariant_basis, (long long)(N + 1) * (N + 1) * nEl, *dxds, *dsdx);
}
void AdjustBoundaryContravariantBasis_SEMQuad_gpu_wrapper(double** dsdx, double** J, int N, int nEl) {
  LAUNCH(k_adjust_boundary_basis, (long long)(N + 1) * 4 * nEl, *dsdx, *J, N);
}
void GradientBR_MappedScalar2D_gpu_wrapper(double** scalar, double** avgBoundary, double** dsdx, double** jacobian,
                                           double** nHat, double** nScale, double** gradF, double** dgMatrix,
                                           double** bMatrix, double** qWeights, int N, int nVar, int nEl) {
  LAUNCH(k_gradient_br, (long long)(N + 1) * (N + 1) * nVar * nEl, *scalar, *avgBoundary, *dsdx, *jacobian, *nHat,
         *nScale, *gradF, *dgMatrix, *bMatrix, *qWeights, N, nVar);
}
void GradientSF_MappedScalar2D_gpu_wrapper(double** scalar, double** dsdx, double** jacobian, double** gradF,
                                           double** dMatrix, int N, int nVar, int nEl) {
  LAUNCH(k_gradient_sf, (long long)(N + 1) * (N + 1) * nVar * nEl, *scalar, *dsdx, *jacobian, *gradF, *dMatrix, N,
         nVar);
}
void JacobianWeight_MappedScalar2D_gpu_wrapper(double** scalar, double** jacobian, int N, int nVar, int nEl) {
  LAUNCH(k_jacobian_weight<1>, (long long)(N + 1) * (N + 1) * nVar * nEl, *scalar, *jacobian, N, nVar);
}
void JacobianWeight_MappedVector2D_gpu_wrapper(double** vector, double** jacobian, int N, int nVar, int nEl) {
  LAUNCH(k_jacobian_weight<2>, 2LL * (N + 1) * (N + 1) * nVar * nEl, *vector, *jacobian, N, nVar);
}
void ContravariantProjection_MappedVector2D_gpu_wrapper(double** vector, double** dsdx, int N, int nVar, int nEl) {
  LAUNCH(k_contravariant_projection, (long long)(N + 1) * (N + 1) * nVar * nEl, *vector, *dsdx, N, nVar);
}
void SideExchange_MappedScalar2D_gpu_wrapper(double** extBoundary, double** boundary, int** sideInfo,
                                             int** elemToRank, int rankId, int offset, int N, int nVar, int nEl) {
  LAUNCH(k_side_exchange<1>, (long long)(N + 1) * nVar * 4 * nEl, *extBoundary, *boundary, *sideInfo,
         elemToRank ? *elemToRank : nullptr, rankId, offset, N, nVar);
}
void SideExchange_MappedVector2D_gpu_wrapper(double** extBoundary, double** boundary, int** sideInfo,
                                             int** elemToRank, int rankId, int offset, int N, int nVar, int nEl) {
  LAUNCH(k_side_exchange<2>, 2LL * (N + 1) * nVar * 4 * nEl, *extBoundary, *boundary, *sideInfo,
         elemToRank ? *elemToRank : nullptr, rankId, offset, N, nVar);
}
void BassiRebaySides_MappedScalar2D_gpu_wrapper(double** avgBoundary, double** boundary, double** extBoundary, int N,
                                                int nVar, int nEl) {
  LAUNCH(k_bassi_rebay, (long long)(N + 1) * nVar * 4 * nEl, *avgBoundary, *boundary, *extBoundary);
}
void UpdateGRK_Model2D_gpu_wrapper(double** grk, double** solution, double** dSdt, double rk_a, double rk_g, double dt,
                                   int nWork, int N, int nVar, int nEl) {
  LAUNCH(k_update_grk, (long long)(N + 1) * (N + 1) * nVar * nEl, *grk, *solution, *dSdt, rk_a, rk_g, dt, nWork, N,
         nVar);
}
void UpdateSolution_Model2D_gpu_wrapper(double** solution, double** dSdt, double dt, int N, int nVar, int nEl) {
  LAUNCH(k_update_solution, (long long)(N + 1) * (N + 1) * nVar * nEl, *solution, *dSdt, dt);
}
void CalculateDSDt_Model2D_gpu_wrapper(double** fluxDivergence, double** source, double** dSdt, int N, int nVar,
                                       int nEl) {
  LAUNCH(k_dsdt, (long long)(N + 1) * (N + 1) * nVar * nEl, *fluxDivergence, *source, *dSdt);
}
void SetBoundaryCondition_LinearShallowWater_gpu_wrapper(double** solution, double** extBoundary, double** nHat,
                                                         int** sideInfo, int N, int nVar, int nEl) {
  LAUNCH(k_lsw_bc, (long long)(N + 1) * 4 * nEl, *solution, *extBoundary, *nHat, *sideInfo, N, nVar);
}
void Source_LinearShallowWater_gpu_wrapper(double** source, double** solution, double** f, int N, int nVar, int nEl) {
  LAUNCH(k_lsw_source, (long long)(N + 1) * (N + 1) * nEl, *source, *solution, *f, N, nVar);
}
void Flux_LinearShallowWater_gpu_wrapper(double** flux, double** solution, double** H, double g, int N, int nVar,
                                         int nEl) {
  LAUNCH(k_lsw_flux, (long long)(N + 1) * (N + 1) * nEl, *flux, *solution, *H, g, N, nVar);
}
void RiemannSolver_LinearShallowWater_gpu_wrapper(double** flux, double** solution, double** extBoundary, double** H,
                                                  double** nHat, double** nScale, double g, int N, int nVar,
                                                  int nEl) {
  LAUNCH(k_lsw_riemann, (long long)(N + 1) * 4 * nEl, *flux, *solution, *extBoundary, *H, *nHat, *nScale, g, N, nVar);
}
void SetBoundaryCondition_ShallowWater_gpu_wrapper(double** solution, double** extBoundary, double** topoBoundary,
                                                   double** nHat, int** sideInfo, int N, int nVar, int nEl) {
  LAUNCH(k_sw_bc, (long long)(N + 1) * 4 * nEl, *solution, *extBoundary, *topoBoundary, *nHat, *sideInfo, N, nVar);
}
void Source_ShallowWater_gpu_wrapper(double** source, double** solution, double** gradH, double fCori, double g, int N,
                                     int nVar, int nEl) {
  LAUNCH(k_sw_source, (long long)(N + 1) * (N + 1) * nEl, *source, *solution, *gradH, fCori, g, N, nVar);
}
void Flux_ShallowWater_gpu_wrapper(double** flux, double** solution, double** velocity, double g, int N, int nVar,
                                   int nEl) {
  LAUNCH(k_sw_flux, (long long)(N + 1) * (N + 1) * nEl, *flux, *solution, *velocity, g, N, nVar);
}
void RiemannSolver_ShallowWater_gpu_wrapper(double** flux, double** solution, double** extBoundary, double** velocity,
                                            double** extVelocity, double** nHat, double** nScale, double g, int N,
                                            int nVar, int nEl) {
  LAUNCH(k_sw_riemann, (long long)(N + 1) * 4 * nEl, *flux, *solution, *extBoundary, *velocity, *extVelocity, *nHat,
         *nScale, g, N, nVar);
}
void PreTendency_ShallowWater_gpu_wrapper(double** solution, double** solutionBoundary, double** velocity,
                                          double** velocityBoundary, int N, int nVar, int nEl) {
  const int P = N + 1;
  LAUNCH(k_sw_velocity, (long long)P * P * nEl, *solution, *velocity, P * P, nVar);
  LAUNCH(k_sw_velocity, (long long)P * 4 * nEl, *solutionBoundary, *velocityBoundary, P, nVar);
}
void Source_CompressibleIdealGas2D_gpu_wrapper(double** source, double** solution, double** environmentalsGradient,
                                               int N, int nVar, int nEl) {
  LAUNCH(k_cig_source, (long long)(N + 1) * (N + 1) * nEl, *source, *solution, *environmentalsGradient, N, nVar);
}
void Flux_CompressibleIdealGas2D_gpu_wrapper(double** flux, double** solution, double** primitive, int N, int nVar,
                                             int nEl) {
  // The signature carries no diagnostics array; rhoH = rhoE + p is formed from
  // the solution and the primitive pressure, as the reference device kernel does.
  LAUNCH(k_cig_flux, (long long)(N + 1) * (N + 1) * nEl, *flux, *solution, *primitive, (const double*)nullptr, N, nVar);
}
void NaiveLLF_CompressibleIdealGas2D_gpu_wrapper(double** flux, double** solution, double** extSolution,
                                                 double** primitive, double** extPrimitive, double** diagnostics,
                                                 double** extDiagnostics, double** nHat, double** nScale, int N,
                                                 int nVar, int nDiag, int nEl) {
  LAUNCH(k_cig_llf, (long long)(N + 1) * 4 * nEl, *flux, *solution, *extSolution, *primitive, *extPrimitive,
         *diagnostics, *extDiagnostics, *nHat, *nScale, N, nVar, nDiag);
}
void SetBoundaryCondition_CompressibleIdealGas2D_gpu_wrapper(
    double** solution, double** extSolution, double** prescribedSolution, double** primitive, double** extPrimitive,
    double** prescribedPrimitive, double** diagnostics, double** extDiagnostics, double** prescribedDiagnostics,
    double** nHat, int** sideInfo, int N, int nVar, int nDiag, int nEl) {
  const long long n = (long long)(N + 1) * 4 * nEl;
  LAUNCH(k_cig_bc, n, *solution, *extSolution, *prescribedSolution, *nHat, *sideInfo, N, nVar, 1);
  LAUNCH(k_cig_bc, n, *primitive, *extPrimitive, *prescribedPrimitive, *nHat, *sideInfo, N, nVar, 1);
  LAUNCH(k_cig_bc, n, *diagnostics, *extDiagnostics, *prescribedDiagnostics, *nHat, *sideInfo, N, nDiag, 0);
}
void CalculateDiagnostics_CompressibleIdealGas2D_gpu_wrapper(double** solution, double** diagnostics,
                                                             double expansionFactor, double R, int N, int nVar,
                                                             int nDiag, int nEl) {
  LAUNCH(k_cig_pointwise, (long long)(N + 1) * (N + 1) * nEl, *solution, *diagnostics, expansionFactor, R, 0, N, nVar,
         nDiag);
}
void ConservativeToPrimitive_CompressibleIdealGas2D_gpu_wrapper(double** solution, double** primitive,
                                                                double expansionFactor, int N, int nVar, int nEl) {
  LAUNCH(k_cig_pointwise, (long long)(N + 1) * (N + 1) * nEl, *solution, *primitive, expansionFactor, 1.0, 1, N, nVar,
         nVar);
}
void ConservativeToEntropy_CompressibleIdealGas2D_gpu_wrapper(double** solution, double** entropy,
                                                              double expansionFactor, int N, int nVar, int nEl) {
  LAUNCH(k_cig_pointwise, (long long)(N + 1) * (N + 1) * nEl, *solution, *entropy, expansionFactor, 1.0, 2, N, nVar,
         nVar);
}

}  // extern "C"

// ---------------------------------------------------------- device geometry
extern "C" int selfgpu_semquad_generate(int N, int nEl, const double* nodeCoords_d, const double* m2m_iMatrix,
                                        const double* dMatrix, const double* bMatrix, double* x_d, double* dxds_d,
                                        double* dsdx_d, double* J_d, double* dsdxB_d, double* JB_d, double* nHat_d,
                                        double* nScale_d, void* stream) {
  if (N < 1 || N > 15 || nEl < 1 || !nodeCoords_d || !m2m_iMatrix || !dMatrix || !bMatrix || !x_d || !dxds_d ||
      !dsdx_d || !J_d || !dsdxB_d || !JB_d || !nHat_d || !nScale_d)
    return set_error(SELFGPU_ERR_ARG, "selfgpu_semquad_generate: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const int P = N + 1;
  // Matrices to the device: iM (0:1,0:N), dM (P*P), bM (P*2)
  double* mats = nullptr;
  const size_t nm = 2 * P + P * P + 2 * P;
  if (cudaMalloc(&mats, nm * sizeof(double)) != cudaSuccess)
    return set_error(SELFGPU_ERR_CUDA, "selfgpu_semquad_generate: cudaMalloc failed");
  cudaMemcpyAsync(mats, m2m_iMatrix, 2 * P * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(mats + 2 * P, dMatrix, P * P * sizeof(double), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(mats + 2 * P + P * P, bMatrix, 2 * P * sizeof(double), cudaMemcpyHostToDevice, st);
  const double *iM = mats, *dM = mats + 2 * P, *bM = mats + 2 * P + P * P;
  const long long nNodes = (long long)P * P * nEl, nFace = (long long)P * 4 * nEl;
  // GenerateFromMesh_SEMQuad: x = GridInterp(nodeCoords), src/SELF_Geometry.f90:393-435
  k_vector_grid_interp<<<blocks_for(2 * nNodes), kThreads, 0, st>>>(iM, nodeCoords_d, x_d, 1, N, 2 * nNodes);
  // CalculateMetricTerms_SEMQuad, src/SELF_Geometry.f90:528-552
  k_vector_gradient<<<blocks_for(nNodes), kThreads, 0, st>>>(dM, x_d, dxds_d, N, nNodes);
  k_determinant<<<blocks_for(nNodes), kThreads, 0, st>>>(dxds_d, J_d, nNodes);
  k_scalar_boundary_interp<<<blocks_for((long long)P * nEl), kThreads, 0, st>>>(bM, J_d, JB_d, N, 1,
                                                                              (long long)P * nEl);
  k_contravariant_basis<<<blocks_for(nNodes), kThreads, 0, st>>>(dxds_d, dsdx_d, nNodes);
  k_multi_boundary_interp<4><<<blocks_for(4LL * P * nEl), kThreads, 0, st>>>(bM, dsdx_d, dsdxB_d, N, 1,
                                                                           4LL * P * nEl);
  k_face_normals<<<blocks_for(nFace), kThreads, 0, st>>>(dsdxB_d, JB_d, nHat_d, nScale_d, N, nFace);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaFree(mats);
  if (e != cudaSuccess) return set_error(SELFGPU_ERR_CUDA, std::string("selfgpu_semquad_generate: ") + cudaGetErrorString(e));
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(SELFGPU_ERR_CUDA, std::string("selfgpu_semquad_generate: ") + cudaGetErrorString(e));
  return SELFGPU_OK;
}
