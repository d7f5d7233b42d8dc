// self_oracle.cpp -- FP64 CPU restatement of SELF's 2-D DGSEM tendency path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA engine in
// self_b200/: only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
// leg may load it.  It is never linked into, or called by, the product path.
//
// Every routine restates the CPU (non-GPU) branch of the reference Fortran with
// the same loop order and the same left-to-right evaluation of each
// expression, in double precision (the reference's -DDOUBLE_PRECISION build,
// src/SELF_Constants.f90:20-26).  Build it with -ffp-contract=off for parity
// (gfortran on x86-64 does not contract to FMA without -march).  Element loops
// may run under OpenMP: the arithmetic inside an element does not depend on the
// thread count, so results are bit-identical for any number of threads.
//
// Layouts are Fortran column-major, node index fastest (src/SELF_Data.f90:565-572,
// src/hip/SELF_HIP_Macros.h:20-38):
//   scalar interior (0:N,0:N,nVar,nEl)      boundary (0:N,nVar,4,nEl)
//   vector interior (2,0:N,0:N,nVar,nEl)    boundary (2,0:N,nVar,4,nEl)
//   tensor interior (2,2,0:N,0:N,nVar,nEl)  boundary (2,2,0:N,nVar,4,nEl)
//   sideInfo (5,4,nEl), 1-based element ids (src/SELF_Mesh.f90:80-88)
// Sides: 1=South 2=East 3=North 4=West (src/SELF_Mesh.f90:42-45).
//
// Parity status: the reference cannot be compiled here (no Fortran compiler,
// hipfort, MPI or HDF5) and its tests hold no numeric golden vectors; this
// restatement is pinned by the mesh fixtures read from the reference's own
// etc/mesh/*.mesh files, by published quadrature values and by the exact
// invariants the reference tests assert (tests/test_oracle_*.py).

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

// src/SELF_Constants.f90:78-84
constexpr int GAUSS = 1, GAUSS_LOBATTO = 2, CHEBYSHEV_GAUSS = 3, CHEBYSHEV_GAUSS_LOBATTO = 4,
              UNIFORM = 5;
// src/hip/SELF_HIP_Macros.h:40-49
constexpr int BC_PRESCRIBED = 100, BC_RADIATION = 101, BC_NONORMALFLOW = 102;
constexpr int NEWTON_MAX = 500;  // src/SELF_Constants.f90:52
static const double PI = 4.0 * std::atan(1.0);  // src/SELF_Constants.f90:41
static const double TOL = DBL_EPSILON;           // src/SELF_Constants.f90:42

using Vec = std::vector<double>;

static const int kOrcMaxP = 16;

// ---------------------------------------------------------------- quadrature
// src/SELF_Quadrature.f90:342-383 (Kopriva Alg. 22)
static void LegendrePolynomial(int N, double x, double& l, double& dl) {
  if (N == 0) {
    l = 1.0;
    dl = 0.0;
  } else if (N == 1) {
    l = x;
    dl = 1.0;
  } else {
    double lnm2 = 1.0, lnm1 = x, dlnm2 = 0.0, dlnm1 = 1.0;
    for (int i = 2; i <= N; ++i) {
      double di = (double)i;
      l = ((2.0 * di - 1.0) * x * lnm1 - (di - 1.0) * lnm2) / di;
      dl = dlnm2 + (2.0 * di - 1.0) * lnm1;
      lnm2 = lnm1;
      lnm1 = l;
      dlnm2 = dlnm1;
      dlnm1 = dl;
    }
  }
}

// src/SELF_Quadrature.f90:390-422 (Kopriva Alg. 24)
static void LegendreQandL(int N, double x, double& q, double& qp, double& lN) {
  double lnm2 = 1.0, lnm1 = x, dlnm2 = 0.0, dlnm1 = 1.0, dlN = 0.0;
  lN = 0.0;
  for (int i = 2; i <= N; ++i) {
    double di = (double)i;
    lN = (2.0 * i - 1.0) / di * x * lnm1 - (di - 1.0) / di * lnm2;
    dlN = dlnm2 + (2.0 * di - 1.0) * lnm1;
    lnm2 = lnm1;
    lnm1 = lN;
    dlnm2 = dlnm1;
    dlnm1 = dlN;
  }
  int i = N + 1;
  double di = (double)i;
  double lN1 = (2.0 * i - 1.0) / di * x * lN - (di - 1.0) / di * lnm2;
  double dlN1 = dlnm2 + (2.0 * di - 1.0) * lnm1;
  q = lN1 - lnm2;
  qp = dlN1 - dlnm2;
}

// src/SELF_Quadrature.f90:201-262.  Quirks kept (hazard H11): the initial
// guess uses 2N+1 in the denominator, the Newton exit test abs(delta) <=
// TOL*x never fires for x < 0 (so those nodes take all 500 iterations), and the
// j loop runs to (N+1)/2 so one mirrored node is overwritten.  The N == 1
// branch reads the output array before it is written; the reference's output
// array is zero-initialised (src/SELF_Memory.f90 Alloc sets hostData = 0), so
// nodes(1) = weights(1) = 0 there, which is reproduced.
static void LegendreGauss(int N, double* nodes, double* weights) {
  Vec xl(N + 1, 0.0), wl(N + 1, 0.0);
  if (N == 0) {
    xl[0] = 0.0;
    wl[0] = 2.0;
  } else if (N == 1) {
    xl[0] = -std::sqrt(1.0 / 3.0);
    wl[0] = 1.0;
    xl[1] = -0.0;  // -nodes(0) with nodes(0) == 0
    wl[1] = 0.0;   // weights(0) == 0
  } else {
    for (int j = 0; j <= (N + 1) / 2; ++j) {
      xl[j] = -std::cos((2.0 * (double)j + 1.0) * PI / (2.0 * (double)N + 1.0));
      double l, dl;
      for (int k = 1; k <= NEWTON_MAX; ++k) {
        LegendrePolynomial(N + 1, xl[j], l, dl);
        double delta = -l / dl;
        xl[j] = xl[j] + delta;
        if (std::fabs(delta) <= TOL * xl[j]) break;
      }
      LegendrePolynomial(N + 1, xl[j], l, dl);
      wl[j] = 2.0 / ((1.0 - xl[j] * xl[j]) * dl * dl);
      wl[N - j] = wl[j];
      xl[N - j] = -xl[j];
    }
  }
  if (std::fmod((double)N, 2.0) == 0.0) {
    double l, dl;
    LegendrePolynomial(N + 1, 0.0, l, dl);
    xl[N / 2] = 0.0;
    wl[N / 2] = 2.0 / (dl * dl);
  }
  for (int j = 0; j <= N; ++j) {
    nodes[j] = xl[j];
    weights[j] = wl[j];
  }
}

// src/SELF_Quadrature.f90:270-335
static void LegendreGaussLobatto(int N, double* nodes, double* weights) {
  Vec xl(N + 1, 0.0), wl(N + 1, 0.0);
  if (N == 1) {
    xl[0] = -1.0;
    wl[0] = 1.0;
    xl[1] = 1.0;
    wl[1] = 1.0;
  } else {
    double dN = (double)N;
    xl[0] = -1.0;
    wl[0] = 2.0 / (dN * (dN + 1.0));
    xl[N] = 1.0;
    wl[N] = wl[0];
    for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
      double dj = (double)j;
      xl[j] = -std::cos((dj + 0.25) * PI / dN - 3.0 / (8.0 * dN * PI * (dj + 0.25)));
      double q, qp, lN;
      for (int k = 1; k <= NEWTON_MAX; ++k) {
        LegendreQandL(N, xl[j], q, qp, lN);
        double delta = -q / qp;
        xl[j] = xl[j] + delta;
        if (std::fabs(delta) <= TOL * xl[j]) break;
      }
      LegendreQandL(N, xl[j], q, qp, lN);
      wl[j] = 2.0 / (dN * (dN + 1.0) * lN * lN);
      wl[N - j] = wl[j];
      xl[N - j] = -xl[j];
    }
  }
  if (std::fmod((double)N, 2.0) == 0.0) {
    double q, qp, lN;
    LegendreQandL(N, 0.0, q, qp, lN);
    double dN = (double)N;
    xl[N / 2] = 0.0;
    wl[N / 2] = 2.0 / (dN * (dN + 1.0) * lN * lN);
  }
  for (int j = 0; j <= N; ++j) {
    nodes[j] = xl[j];
    weights[j] = wl[j];
  }
}

// src/SELF_Quadrature.f90:148-197
static void ChebyshevQuad(int N, int type, double* nodes, double* weights) {
  double dN = (double)N;
  if (type == CHEBYSHEV_GAUSS_LOBATTO) {
    for (int j = 0; j <= N; ++j) {
      weights[j] = PI / dN;
      nodes[j] = -std::cos(PI * (double)j / dN);
    }
    weights[0] = weights[0] * 0.5;
    weights[N] = weights[N] * 0.5;
  } else {
    for (int j = 0; j <= N; ++j) {
      weights[j] = PI / (dN + 1.0);
      nodes[j] = -std::cos(PI * (2.0 * (double)j + 1.0) / (2.0 * dN + 2.0));
    }
  }
}

// src/SELF_SupportRoutines.f90:76-96
static bool AlmostEqual(double a, double b) {
  if (a == 0.0 || b == 0.0) return std::fabs(a - b) <= DBL_EPSILON;
  return (std::fabs(a - b) <= DBL_EPSILON * std::fabs(a)) ||
         (std::fabs(a - b) <= DBL_EPSILON * std::fabs(b));
}

// src/SELF_SupportRoutines.f90:502-520
static void UniformPoints(double a, double b, int first, int last, double* x) {
  double dx = (b - a) / (double)(last - first);
  for (int i = first; i <= last; ++i) x[i - first] = a + dx * (double)(i - first);
}

// ------------------------------------------------------------------ Lagrange
// src/SELF_Lagrange.f90:25-192, 521-615, 2542-2774
struct Lagrange {
  int N = 0, M = 0, ctrlType = 0, tgtType = 0;
  Vec ctrl, tgt, bw, qw;
  Vec iM;   // iMatrix%hostData(0:N,0:M): iM[ii + (N+1)*m]
  Vec dM;   // dMatrix%hostData(0:N,0:N): dM[ii + P*i]
  Vec dgM;  // dgMatrix%hostData(0:N,0:N)
  Vec bM;   // bMatrix%hostData(0:N,0:1): bM[ii + P*side]

  void init(int N_, int ctrlType_, int M_, int tgtType_) {
    N = N_;
    M = M_;
    ctrlType = ctrlType_;
    tgtType = tgtType_;
    int P = N + 1, Q = M + 1;
    ctrl.assign(P, 0.0);
    tgt.assign(Q, 0.0);
    bw.assign(P, 0.0);
    qw.assign(P, 0.0);
    iM.assign((size_t)P * Q, 0.0);
    dM.assign((size_t)P * P, 0.0);
    dgM.assign((size_t)P * P, 0.0);
    bM.assign((size_t)P * 2, 0.0);
    if (ctrlType == GAUSS) {
      LegendreGauss(N, ctrl.data(), qw.data());
    } else if (ctrlType == GAUSS_LOBATTO) {
      LegendreGaussLobatto(N, ctrl.data(), qw.data());
    } else if (ctrlType == CHEBYSHEV_GAUSS || ctrlType == CHEBYSHEV_GAUSS_LOBATTO) {
      ChebyshevQuad(N, ctrlType, ctrl.data(), qw.data());
    } else if (ctrlType == UNIFORM) {
      UniformPoints(-1.0, 1.0, 0, N, ctrl.data());
      for (int i = 0; i < P; ++i) qw[i] = 2.0 / (double)N;
    }
    Vec q(Q, 0.0);
    if (tgtType == GAUSS) {
      LegendreGauss(M, tgt.data(), q.data());
    } else if (tgtType == GAUSS_LOBATTO) {
      LegendreGaussLobatto(M, tgt.data(), q.data());
    } else if (tgtType == UNIFORM) {
      UniformPoints(-1.0, 1.0, 0, M, tgt.data());
    }
    barycentric();
    interpolationMatrix();
    derivativeMatrix();
    Vec l(P);
    lagrangePolys(-1.0, l.data());
    for (int i = 0; i < P; ++i) bM[i] = l[i];
    lagrangePolys(1.0, l.data());
    for (int i = 0; i < P; ++i) bM[i + P] = l[i];
  }

  // Kopriva Alg. 30, src/SELF_Lagrange.f90:2542-2570
  void barycentric() {
    Vec b(N + 1, 1.0);
    for (int j = 1; j <= N; ++j)
      for (int i = 0; i <= j - 1; ++i) {
        b[i] = b[i] * (ctrl[i] - ctrl[j]);
        b[j] = b[j] * (ctrl[j] - ctrl[i]);
      }
    for (int j = 0; j <= N; ++j) bw[j] = 1.0 / b[j];
  }

  // Kopriva Alg. 32, src/SELF_Lagrange.f90:2582-2637
  void interpolationMatrix() {
    int P = N + 1;
    for (int row = 0; row <= M; ++row) {
      Vec r(P, 0.0);
      bool match = false;
      for (int col = 0; col <= N; ++col) {
        r[col] = 0.0;
        if (AlmostEqual(tgt[row], ctrl[col])) {
          match = true;
          r[col] = 1.0;
        }
      }
      if (!match) {
        double t1 = 0.0;
        for (int col = 0; col <= N; ++col) {
          double t2 = bw[col] / (tgt[row] - ctrl[col]);
          r[col] = t2;
          t1 = t1 + t2;
        }
        for (int col = 0; col <= N; ++col) r[col] = r[col] / t1;
      }
      for (int col = 0; col <= N; ++col) iM[col + (size_t)P * row] = r[col];
    }
  }

  // Kopriva Alg. 37, src/SELF_Lagrange.f90:2650-2708
  void derivativeMatrix() {
    int P = N + 1;
    Vec dm((size_t)P * P, 0.0), dg((size_t)P * P, 0.0);
    auto D = [&](int r, int c) -> double& { return dm[r + (size_t)P * c]; };
    auto G = [&](int r, int c) -> double& { return dg[r + (size_t)P * c]; };
    for (int row = 0; row <= N; ++row) {
      D(row, row) = 0.0;
      for (int col = 0; col <= N; ++col) {
        if (col != row) {
          D(row, col) = bw[col] / (bw[row] * (ctrl[row] - ctrl[col]));
          D(row, row) = D(row, row) - D(row, col);
        }
      }
    }
    for (int row = 0; row <= N; ++row)
      for (int col = 0; col <= N; ++col) G(row, col) = -D(col, row) * qw[col] / qw[row];
    for (int row = 0; row <= N; ++row)
      for (int col = 0; col <= N; ++col) {
        dM[row + (size_t)P * col] = D(col, row);
        dgM[row + (size_t)P * col] = G(col, row);
      }
  }

  // Kopriva Alg. 34, src/SELF_Lagrange.f90:2720-2774
  void lagrangePolys(double sE, double* out) {
    int P = N + 1;
    Vec l(P, 0.0);
    bool match = false;
    for (int j = 0; j <= N; ++j) {
      l[j] = 0.0;
      if (AlmostEqual(sE, ctrl[j])) {
        l[j] = 1.0;
        match = true;
      }
    }
    if (!match) {
      double t1 = 0.0;
      for (int j = 0; j <= N; ++j) {
        double t2 = bw[j] / (sE - ctrl[j]);
        l[j] = t2;
        t1 = t1 + t2;
      }
      for (int j = 0; j <= N; ++j) l[j] = l[j] / t1;
    }
    for (int j = 0; j < P; ++j) out[j] = l[j];
  }
};

// ---------------------------------------------------------- tensor-product ops
#define SC(i, j, v, e) ((i) + P * ((j) + P * ((v) + (size_t)nVar * (e))))
#define SCB(i, v, s, e) ((i) + P * ((v) + (size_t)nVar * ((s) + 4 * (size_t)(e))))
#define VE(d, i, j, v, e) ((d) + 2 * SC(i, j, v, e))
#define VEB(d, i, v, s, e) ((d) + 2 * SCB(i, v, s, e))
#define TE(r, c, i, j, v, e) ((r) + 2 * ((c) + 2 * SC(i, j, v, e)))
#define TEB(r, c, i, v, s, e) ((r) + 2 * ((c) + 2 * SCB(i, v, s, e)))
#define OMP_FOR _Pragma("omp parallel for schedule(static)")

// src/SELF_Lagrange.f90:2241-2270
static void ScalarBoundaryInterp2D(const double* bM, const double* f, double* fb, int N, int nVar,
                                   int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int i = 0; i < P; ++i) {
        double b1 = 0, b2 = 0, b3 = 0, b4 = 0;
        for (int ii = 0; ii < P; ++ii) {
          b1 = b1 + bM[ii] * f[SC(i, ii, v, e)];
          b2 = b2 + bM[ii + P] * f[SC(ii, i, v, e)];
          b3 = b3 + bM[ii + P] * f[SC(i, ii, v, e)];
          b4 = b4 + bM[ii] * f[SC(ii, i, v, e)];
        }
        fb[SCB(i, v, 0, e)] = b1;
        fb[SCB(i, v, 1, e)] = b2;
        fb[SCB(i, v, 2, e)] = b3;
        fb[SCB(i, v, 3, e)] = b4;
      }
}

// src/SELF_Lagrange.f90:2284-2316
static void VectorBoundaryInterp2D(const double* bM, const double* f, double* fb, int N, int nVar,
                                   int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int i = 0; i < P; ++i) {
        double b[2][4] = {{0}};
        for (int ii = 0; ii < P; ++ii)
          for (int d = 0; d < 2; ++d) {
            b[d][0] = b[d][0] + bM[ii] * f[VE(d, i, ii, v, e)];
            b[d][1] = b[d][1] + bM[ii + P] * f[VE(d, ii, i, v, e)];
            b[d][2] = b[d][2] + bM[ii + P] * f[VE(d, i, ii, v, e)];
            b[d][3] = b[d][3] + bM[ii] * f[VE(d, ii, i, v, e)];
          }
        for (int d = 0; d < 2; ++d)
          for (int s = 0; s < 4; ++s) fb[VEB(d, i, v, s, e)] = b[d][s];
      }
}

// src/SELF_Lagrange.f90:2330-2366
static void TensorBoundaryInterp2D(const double* bM, const double* f, double* fb, int N, int nVar,
                                   int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int i = 0; i < P; ++i) {
        double b[2][2][4] = {{{0}}};
        for (int ii = 0; ii < P; ++ii)
          for (int c = 0; c < 2; ++c)
            for (int r = 0; r < 2; ++r) {
              b[r][c][0] = b[r][c][0] + bM[ii] * f[TE(r, c, i, ii, v, e)];
              b[r][c][1] = b[r][c][1] + bM[ii + P] * f[TE(r, c, ii, i, v, e)];
              b[r][c][2] = b[r][c][2] + bM[ii + P] * f[TE(r, c, i, ii, v, e)];
              b[r][c][3] = b[r][c][3] + bM[ii] * f[TE(r, c, ii, i, v, e)];
            }
        for (int c = 0; c < 2; ++c)
          for (int r = 0; r < 2; ++r)
            for (int s = 0; s < 4; ++s) fb[TEB(r, c, i, v, s, e)] = b[r][c][s];
      }
}

// src/SELF_Lagrange.f90:741-789 (iM is iMatrix%hostData(0:N,0:M))
static void ScalarGridInterp2D(const double* iM, const double* f, double* fo, int N, int M,
                               int nVar, int nEl) {
  int P = N + 1, Q = M + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < Q; ++j)
        for (int i = 0; i < Q; ++i) {
          double fij = 0.0;
          for (int jj = 0; jj < P; ++jj) {
            double fi = 0.0;
            for (int ii = 0; ii < P; ++ii)
              fi = fi + f[ii + P * (jj + P * (v + (size_t)nVar * e))] * iM[ii + (size_t)P * i];
            fij = fij + fi * iM[jj + (size_t)P * j];
          }
          fo[i + Q * (j + Q * (v + (size_t)nVar * e))] = fij;
        }
}

// src/SELF_Lagrange.f90:824-875
static void VectorGridInterp2D(const double* iM, const double* f, double* fo, int N, int M,
                               int nVar, int nEl) {
  int P = N + 1, Q = M + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < Q; ++j)
        for (int i = 0; i < Q; ++i) {
          double o[2] = {0.0, 0.0};
          for (int jj = 0; jj < P; ++jj) {
            double fi[2] = {0.0, 0.0};
            for (int ii = 0; ii < P; ++ii)
              for (int d = 0; d < 2; ++d)
                fi[d] = fi[d] + f[d + 2 * (ii + P * (jj + P * (v + (size_t)nVar * e)))] *
                                    iM[ii + (size_t)P * i];
            for (int d = 0; d < 2; ++d) o[d] = o[d] + fi[d] * iM[jj + (size_t)P * j];
          }
          for (int d = 0; d < 2; ++d) fo[d + 2 * (i + Q * (j + Q * (v + (size_t)nVar * e)))] = o[d];
        }
}

// src/SELF_Lagrange.f90:1424-1463
static void VectorGradient2D(const double* dM, const double* f, double* gf, int N, int nVar,
                             int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double g11 = 0, g21 = 0, g12 = 0, g22 = 0;
          for (int ii = 0; ii < P; ++ii) {
            g11 = g11 + dM[ii + P * i] * f[VE(0, ii, j, v, e)];
            g21 = g21 + dM[ii + P * i] * f[VE(1, ii, j, v, e)];
            g12 = g12 + dM[ii + P * j] * f[VE(0, i, ii, v, e)];
            g22 = g22 + dM[ii + P * j] * f[VE(1, i, ii, v, e)];
          }
          gf[TE(0, 0, i, j, v, e)] = g11;
          gf[TE(1, 0, i, j, v, e)] = g21;
          gf[TE(0, 1, i, j, v, e)] = g12;
          gf[TE(1, 1, i, j, v, e)] = g22;
        }
}

// src/SELF_Lagrange.f90:1589-1625 (weak form with surface lift)
static void VectorDGDivergence2D(const double* dgM, const double* bM, const double* qw,
                                 const double* f, const double* bf, double* df, int N, int nVar,
                                 int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double d = 0.0;
          for (int ii = 0; ii < P; ++ii)
            d = d + dgM[ii + P * i] * f[VE(0, ii, j, v, e)] + dgM[ii + P * j] * f[VE(1, i, ii, v, e)];
          d = d + (bM[i + P] * bf[SCB(j, v, 1, e)] + bM[i] * bf[SCB(j, v, 3, e)]) / qw[i] +
              (bM[j + P] * bf[SCB(i, v, 2, e)] + bM[j] * bf[SCB(i, v, 0, e)]) / qw[j];
          df[SC(i, j, v, e)] = d;
        }
}

// src/SELF_MappedData.f90:1235-1268 (division kept, hazard H12)
static void JacobianWeightScalar(double* f, const double* J, int N, int nVar, int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) f[SC(i, j, v, e)] = f[SC(i, j, v, e)] / J[i + P * (j + P * (size_t)e)];
}

// src/SELF_MappedData.f90:2220-2269
static void ContravariantProjection(double* f, const double* dsdx, int N, int nVar, int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          size_t g = (size_t)4 * (i + P * (j + P * (size_t)e));
          double Fx = f[VE(0, i, j, v, e)], Fy = f[VE(1, i, j, v, e)];
          f[VE(0, i, j, v, e)] = dsdx[g + 0] * Fx + dsdx[g + 1] * Fy;  // dsdx(1,1), dsdx(2,1)
          f[VE(1, i, j, v, e)] = dsdx[g + 2] * Fx + dsdx[g + 3] * Fy;  // dsdx(1,2), dsdx(2,2)
        }
}

// src/SELF_MappedData.f90:834-917 (single rank: every neighbour is local)
static void SideExchangeScalar(double* ext, const double* bnd, const int* sideInfo, int N,
                               int nVar, int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e1 = 0; e1 < nEl; ++e1)
    for (int s1 = 0; s1 < 4; ++s1) {
      const int* si = sideInfo + 5 * (s1 + 4 * (size_t)e1);
      int e2 = si[2] - 1, s2 = si[3] / 10, flip = si[3] - s2 * 10, bcid = si[4];
      if (bcid != 0) continue;
      for (int v = 0; v < nVar; ++v)
        for (int i1 = 0; i1 < P; ++i1) {
          int i2 = (flip == 0) ? i1 : N - i1;
          if (flip == 0 || flip == 1) ext[SCB(i1, v, s1, e1)] = bnd[SCB(i2, v, s2 - 1, e2)];
        }
    }
}

// src/SELF_MappedData.f90:1870-1958
static void SideExchangeVector(double* ext, const double* bnd, const int* sideInfo, int N,
                               int nVar, int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e1 = 0; e1 < nEl; ++e1)
    for (int s1 = 0; s1 < 4; ++s1) {
      const int* si = sideInfo + 5 * (s1 + 4 * (size_t)e1);
      int e2 = si[2] - 1, s2 = si[3] / 10, flip = si[3] - s2 * 10, bcid = si[4];
      if (bcid != 0) continue;
      for (int v = 0; v < nVar; ++v)
        for (int i1 = 0; i1 < P; ++i1) {
          int i2 = (flip == 0) ? i1 : N - i1;
          if (flip == 0 || flip == 1)
            for (int d = 0; d < 2; ++d) ext[VEB(d, i1, v, s1, e1)] = bnd[VEB(d, i2, v, s2 - 1, e2)];
        }
    }
}

// src/SELF_MappedData.f90:919-953
static void BassiRebaySides(double* avg, const double* bnd, const double* ext, int N, int nVar,
                            int nEl) {
  size_t n = (size_t)(N + 1) * nVar * 4 * nEl;
  for (size_t k = 0; k < n; ++k) avg[k] = 0.5 * (bnd[k] + ext[k]);
}

// src/SELF_MappedData.f90:1080-1149 (strong form, dMatrix)
static void GradientSF(const double* f, const double* dsdx, const double* J, double* gradF,
                       const double* dM, int N, int nVar, int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double gx = 0.0, gy = 0.0;
          for (int ii = 0; ii < P; ++ii) {
            size_t a = 4 * (ii + P * (j + P * (size_t)e)), b = 4 * (i + P * (ii + P * (size_t)e));
            double f1 = f[SC(ii, j, v, e)] * dsdx[a + 0];
            double f2 = f[SC(i, ii, v, e)] * dsdx[b + 2];
            gx = gx + dM[ii + P * i] * f1 + dM[ii + P * j] * f2;
            f1 = f[SC(ii, j, v, e)] * dsdx[a + 1];
            f2 = f[SC(i, ii, v, e)] * dsdx[b + 3];
            gy = gy + dM[ii + P * i] * f1 + dM[ii + P * j] * f2;
          }
          double Jij = J[i + P * (j + P * (size_t)e)];
          gradF[VE(0, i, j, v, e)] = gx / Jij;
          gradF[VE(1, i, j, v, e)] = gy / Jij;
        }
}

// src/SELF_MappedData.f90:955-1078 (BR1: weak form, dgMatrix, averaged traces)
static void GradientBR(const double* f, const double* avgB, const double* dsdx, const double* J,
                       const double* nHat, const double* nScale, double* gradF, const double* dgM,
                       const double* bM, const double* qw, int N, int nVar, int nEl) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double gx = 0.0, gy = 0.0;
          for (int ii = 0; ii < P; ++ii) {
            size_t a = 4 * (ii + P * (j + P * (size_t)e)), b = 4 * (i + P * (ii + P * (size_t)e));
            double f1 = f[SC(ii, j, v, e)] * dsdx[a + 0];
            double f2 = f[SC(i, ii, v, e)] * dsdx[b + 2];
            gx = gx + dgM[ii + P * i] * f1 + dgM[ii + P * j] * f2;
            f1 = f[SC(ii, j, v, e)] * dsdx[a + 1];
            f2 = f[SC(i, ii, v, e)] * dsdx[b + 3];
            gy = gy + dgM[ii + P * i] * f1 + dgM[ii + P * j] * f2;
          }
          auto nh = [&](int d, int k, int s) { return nHat[d + 2 * (k + P * (s + 4 * (size_t)e))]; };
          auto ns = [&](int k, int s) { return nScale[k + P * (s + 4 * (size_t)e)]; };
          auto av = [&](int k, int s) { return avgB[SCB(k, v, s, e)]; };
          double f1 = av(j, 1) * nh(0, j, 1) * ns(j, 1);
          double f2 = av(j, 3) * nh(0, j, 3) * ns(j, 3);
          gx = gx + (f1 * bM[i + P] + f2 * bM[i]) / qw[i];
          f1 = av(i, 2) * nh(0, i, 2) * ns(i, 2);
          f2 = av(i, 0) * nh(0, i, 0) * ns(i, 0);
          gx = gx + (f1 * bM[j + P] + f2 * bM[j]) / qw[j];
          f1 = av(j, 1) * nh(1, j, 1) * ns(j, 1);
          f2 = av(j, 3) * nh(1, j, 3) * ns(j, 3);
          gy = gy + (f1 * bM[i + P] + f2 * bM[i]) / qw[i];
          f1 = av(i, 2) * nh(1, i, 2) * ns(i, 2);
          f2 = av(i, 0) * nh(1, i, 0) * ns(i, 0);
          gy = gy + (f1 * bM[j + P] + f2 * bM[j]) / qw[j];
          double Jij = J[i + P * (j + P * (size_t)e)];
          gradF[VE(0, i, j, v, e)] = gx / Jij;
          gradF[VE(1, i, j, v, e)] = gy / Jij;
        }
}

// src/SELF_Data.f90:1570-1607
static void Determinant2D(const double* t, double* det, int N, int nVar, int nEl) {
  int P = N + 1;
  for (int e = 0; e < nEl; ++e)
    for (int v = 0; v < nVar; ++v)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i)
          det[SC(i, j, v, e)] = t[TE(0, 0, i, j, v, e)] * t[TE(1, 1, i, j, v, e)] -
                                t[TE(0, 1, i, j, v, e)] * t[TE(1, 0, i, j, v, e)];
}

// ------------------------------------------------- artificial-viscosity closure
// Not part of the reference: the shock closure the CompressibleIdealGas2D
// tendency gains for discontinuous data.  The pieces it is built from are the
// reference's own operators: BassiRebaySides + GradientBR (src/SELF_MappedData.f90:
// 919-1078), VectorBoundaryInterp (src/SELF_Lagrange.f90:2284-2316),
// SideExchange (src/SELF_MappedData.f90:1870-1958) and the diffusive flux
// templates of Advection2D (src/models/hip/SELF_Advection2D.cpp:66-95, :140-175),
// generalised from one diffusivity to one viscosity per element.  Physical
// sides carry no viscous flux (no diffusion through walls or open boundaries).
//
// Modal decay indicator: Persson & Peraire, "Sub-cell shock capturing for
// discontinuous Galerkin methods", AIAA 2006-112.  With orthonormal Legendre
// modes c_kl of the density, S = sum_{max(k,l)=N} c_kl^2 / sum c_kl^2,
// s = log10 S and the activation a(s) = 0 below s0 - kappa, 1 above
// s0 + kappa, (1 + sin(pi (s - s0) / (2 kappa))) / 2 between.  The element
// viscosity is nu = a * c_av * h / N * lambda, lambda = max over nodes of
// |u| + c and h = sqrt(element area).

// T(k,i) = w_i Lt_k(x_i), Lt_k = sqrt((2k+1)/2) L_k: c = T q T^T for nodal q on
// Gauss nodes (exact: the products have degree <= 2N).
static void ModalMatrix(int N, const double* x, const double* w, double* T) {
  int P = N + 1;
  for (int i = 0; i < P; ++i)
    for (int k = 0; k < P; ++k) {
      double l, dl;
      LegendrePolynomial(k, x[i], l, dl);
      T[k + P * i] = (std::sqrt((2.0 * k + 1.0) / 2.0) * l) * w[i];
    }
}

// c[k + P l] = sum_j T(l,j) sum_i T(k,i) q(i,j); q is one element's (P,P) block.
static void ModalCoefficients(const double* T, const double* q, double* c, int P) {
  double t[kOrcMaxP * kOrcMaxP];
  for (int j = 0; j < P; ++j)
    for (int k = 0; k < P; ++k) {
      double acc = 0.0;
      for (int i = 0; i < P; ++i) acc = acc + T[k + P * i] * q[i + P * j];
      t[k + P * j] = acc;
    }
  for (int l = 0; l < P; ++l)
    for (int k = 0; k < P; ++k) {
      double acc = 0.0;
      for (int j = 0; j < P; ++j) acc = acc + T[l + P * j] * t[k + P * j];
      c[k + P * l] = acc;
    }
}

static double ModalDecayActivation(const double* c, int P, double s0, double kappa) {
  int N = P - 1;
  double top = 0.0, total = 0.0;
  for (int l = 0; l < P; ++l)
    for (int k = 0; k < P; ++k) {
      double e = c[k + P * l] * c[k + P * l];
      total = total + e;
      if (k == N || l == N) top = top + e;
    }
  if (!(top > 0.0) || !(total > 0.0)) return 0.0;
  double sv = std::log10(top / total);
  if (sv < s0 - kappa) return 0.0;
  if (sv > s0 + kappa) return 1.0;
  return 0.5 * (1.0 + std::sin(PI * (sv - s0) / (2.0 * kappa)));
}

// 18 features of one variable's modes: the energy fractions of the six highest
// shells max(k,l) = m, of the six highest xi-degrees k and of the six highest
// eta-degrees l (m, k, l = N-5..N), each mapped to (log10(max(E/Et, 1e-16)) + 8) / 8.
static void ModalFeatures(const double* c, int P, double* f) {
  int N = P - 1;
  double total = 0.0, sh[kOrcMaxP] = {0}, ex[kOrcMaxP] = {0}, ey[kOrcMaxP] = {0};
  for (int l = 0; l < P; ++l)
    for (int k = 0; k < P; ++k) {
      double e = c[k + P * l] * c[k + P * l];
      total = total + e;
      int m = k > l ? k : l;
      sh[m] = sh[m] + e;
      ex[k] = ex[k] + e;
      ey[l] = ey[l] + e;
    }
  for (int r = 0; r < 6; ++r) {
    int m = N - 5 + r;
    double fr[3] = {sh[m], ex[m], ey[m]};
    for (int g = 0; g < 3; ++g) {
      double q = total > 0.0 ? fr[g] / total : 0.0;
      if (q < 1e-16) q = 1e-16;
      f[r + 6 * g] = (std::log10(q) + 8.0) / 8.0;
    }
  }
}

// ---------------------------------------------------------------------- mesh
// Structured quadrilateral generator (the reference reads 2-D meshes only from
// HOPr HDF5 files, src/SELF_Mesh.f90:852-1016; hazard H10).  Conventions follow
// src/SELF_Mesh.f90:30-90: corner nodes CN1..CN4 counter-clockwise from
// south-west, sideInfo(1:5,s,e) = (type, global side id, neighbour element,
// 10*neighbour side + flip, bcid).  Periodic neighbours carry bcid = 0 (H9) and
// share global node ids, so RecalculateFlip sees them as matching.  A per-
// element rotation (quarter turns) relabels an element's corners, which is how
// tests reach flip = 1 sides.
static const int CGNSCorner[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};  // nGeo = 1
static const int CGNSSide[4][2] = {{1, 2}, {2, 3}, {4, 3}, {1, 4}};    // src/SELF_Mesh.f90:641-644

struct Mesh2D {
  int nElem = 0, nGeo = 1;
  std::vector<int> sideInfo;       // (5,4,nEl)
  Vec nodeCoords;                  // (2,0:nGeo,0:nGeo,nEl)
  std::vector<int> globalNodeIDs;  // (0:nGeo,0:nGeo,nEl)

  // src/SELF_Mesh.f90:1018-1174 (serial path)
  void RecalculateFlip() {
    std::vector<int> nid1(2 * 4 * nElem, 0), nid2(2 * 4 * nElem, 0);
    int G = nGeo + 1;
    for (int e1 = 0; e1 < nElem; ++e1)
      for (int s1 = 0; s1 < 4; ++s1) {
        int* si = &sideInfo[5 * (s1 + 4 * e1)];
        int e2 = si[2] - 1, s2 = si[3] / 10, bcid = si[4];
        if (bcid != 0) continue;
        for (int l = 0; l < 2; ++l) {
          int c1 = CGNSSide[s1][l] - 1, c2 = CGNSSide[s2 - 1][l] - 1;
          int i = CGNSCorner[c1][0] * nGeo, j = CGNSCorner[c1][1] * nGeo;
          nid1[l + 2 * (s1 + 4 * e1)] = globalNodeIDs[i + G * (j + G * e1)];
          i = CGNSCorner[c2][0] * nGeo;
          j = CGNSCorner[c2][1] * nGeo;
          nid2[l + 2 * (s1 + 4 * e1)] = globalNodeIDs[i + G * (j + G * e2)];
        }
      }
    for (int e1 = 0; e1 < nElem; ++e1)
      for (int s1 = 0; s1 < 4; ++s1) {
        int* si = &sideInfo[5 * (s1 + 4 * e1)];
        int s2 = si[3] / 10, bcid = si[4];
        if (bcid != 0) continue;
        int sum = 0;
        for (int l = 0; l < 2; ++l)
          sum += std::abs(nid1[l + 2 * (s1 + 4 * e1)] - nid2[l + 2 * (s1 + 4 * e1)]);
        si[3] = (sum == 0) ? 10 * s2 : 10 * s2 + 1;
      }
  }

  // src/SELF_Mesh.f90:695-719
  void ResetBoundaryConditionType(int bcid) {
    for (int e = 0; e < nElem; ++e)
      for (int s = 0; s < 4; ++s)
        if (sideInfo[2 + 5 * (s + 4 * e)] == 0) sideInfo[4 + 5 * (s + 4 * e)] = bcid;
  }

  void Structured(int nx, int ny, double x0, double x1, double y0, double y1, int perX, int perY,
                  double amp, int bcid, const int* rot) {
    nGeo = 1;
    nElem = nx * ny;
    sideInfo.assign(5 * 4 * nElem, 0);
    nodeCoords.assign(2 * 4 * nElem, 0.0);
    globalNodeIDs.assign(4 * nElem, 0);
    double dx = (x1 - x0) / (double)nx, dy = (y1 - y0) / (double)ny;
    double h = std::min(dx, dy);
    auto nodeX = [&](int ix, int iy, double* p) {
      p[0] = x0 + dx * (double)ix;
      p[1] = y0 + dy * (double)iy;
      if (amp != 0.0 && ix > 0 && ix < nx && iy > 0 && iy < ny) {
        double d = amp * h * std::sin(2.0 * PI * (p[0] - x0) / (x1 - x0)) *
                   std::sin(2.0 * PI * (p[1] - y0) / (y1 - y0));
        p[0] += d;
        p[1] += d;
      }
    };
    int nnx = perX ? nx : nx + 1;
    int nny = perY ? ny : ny + 1;
    auto nodeId = [&](int ix, int iy) {
      if (perX) ix %= nx;
      if (perY) iy %= ny;
      return 1 + ix + nnx * iy;
    };
    (void)nny;
    // corner k (0..3 = SW,SE,NE,NW) of the unrotated element
    const int off[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        int e = ix + nx * iy;
        int r = rot ? (((rot[e] % 4) + 4) % 4) : 0;
        for (int c = 0; c < 4; ++c) {
          int oc = (c + r) % 4;  // local corner c sits at unrotated corner oc
          int gx = ix + off[oc][0], gy = iy + off[oc][1];
          int i = CGNSCorner[c][0], j = CGNSCorner[c][1];
          nodeX(gx, gy, &nodeCoords[2 * (i + 2 * (j + 2 * e))]);
          globalNodeIDs[i + 2 * (j + 2 * e)] = nodeId(gx, gy);
        }
      }
    // Connectivity: sides on the same grid edge (orientation and lower-left
    // grid node, wrapped where periodic) are neighbours; edges are numbered in
    // the order of their corner-id pairs.  (Corner ids alone cannot separate
    // the two edges of a periodic row one or two elements wide.)
    std::map<std::tuple<int, int, int>, std::vector<std::pair<int, int>>> faces;
    auto corner = [&](int e, int c) {
      return globalNodeIDs[CGNSCorner[c][0] + 2 * (CGNSCorner[c][1] + 2 * e)];
    };
    auto edge = [&](int e, int s) {
      int ix = e % nx, iy = e / nx;
      int r = rot ? (((rot[e] % 4) + 4) % 4) : 0;
      int ka = (CGNSSide[s][0] - 1 + r) % 4, kb = (CGNSSide[s][1] - 1 + r) % 4;
      int xa = ix + off[ka][0], ya = iy + off[ka][1], xb = ix + off[kb][0], yb = iy + off[kb][1];
      int gx = std::min(xa, xb), gy = std::min(ya, yb);
      if (perX) gx %= nx;
      if (perY) gy %= ny;
      return 2 * (gx + (nx + 1) * gy) + (xa == xb ? 1 : 0);
    };
    for (int e = 0; e < nElem; ++e)
      for (int s = 0; s < 4; ++s) {
        int a = corner(e, CGNSSide[s][0] - 1), b = corner(e, CGNSSide[s][1] - 1);
        faces[{std::min(a, b), std::max(a, b), edge(e, s)}].push_back({e, s});
      }
    int gid = 0;
    for (auto& kv : faces) {
      ++gid;
      auto& v = kv.second;
      if (v.size() == 2) {
        for (int k = 0; k < 2; ++k) {
          int e = v[k].first, s = v[k].second, e2 = v[1 - k].first, s2 = v[1 - k].second;
          int* si = &sideInfo[5 * (s + 4 * e)];
          si[0] = 1;
          si[1] = (k == 0) ? gid : -gid;
          si[2] = e2 + 1;
          si[3] = 10 * (s2 + 1);
          si[4] = 0;
        }
      } else {
        for (auto& es : v) {
          int* si = &sideInfo[5 * (es.second + 4 * es.first)];
          si[0] = 1;
          si[1] = gid;
          si[2] = 0;
          si[3] = 0;
          si[4] = bcid;
        }
      }
    }
    RecalculateFlip();
  }
};

// ------------------------------------------------------------------ geometry
// src/SELF_Geometry.f90:38-61, 393-582
struct SEMQuad {
  int N = 0, nEl = 0;
  Vec x, xB, dxds, dxdsB, dsdx, dsdxB, J, JB, nHat, nScale;

  void Generate(const Lagrange& interp, const Mesh2D& mesh) {
    N = interp.N;
    nEl = mesh.nElem;
    int P = N + 1;
    size_t n = (size_t)P * P * nEl, nb = (size_t)P * 4 * nEl;
    x.assign(2 * n, 0.0);
    xB.assign(2 * nb, 0.0);
    dxds.assign(4 * n, 0.0);
    dxdsB.assign(4 * nb, 0.0);
    dsdx.assign(4 * n, 0.0);
    dsdxB.assign(4 * nb, 0.0);
    J.assign(n, 0.0);
    JB.assign(nb, 0.0);
    nHat.assign(2 * nb, 0.0);
    nScale.assign(nb, 0.0);
    Lagrange m2m;
    m2m.init(mesh.nGeo, UNIFORM, N, interp.ctrlType);  // GenerateFromMesh_SEMQuad
    VectorGridInterp2D(m2m.iM.data(), mesh.nodeCoords.data(), x.data(), mesh.nGeo, N, 1, nEl);
    VectorBoundaryInterp2D(interp.bM.data(), x.data(), xB.data(), N, 1, nEl);
    // CalculateMetricTerms_SEMQuad
    VectorGradient2D(interp.dM.data(), x.data(), dxds.data(), N, 1, nEl);
    TensorBoundaryInterp2D(interp.bM.data(), dxds.data(), dxdsB.data(), N, 1, nEl);
    Determinant2D(dxds.data(), J.data(), N, 1, nEl);
    ScalarBoundaryInterp2D(interp.bM.data(), J.data(), JB.data(), N, 1, nEl);
    // CalculateContravariantBasis_SEMQuad
    for (size_t k = 0; k < n; ++k) {
      dsdx[4 * k + 0] = dxds[4 * k + 3];
      dsdx[4 * k + 1] = -dxds[4 * k + 2];
      dsdx[4 * k + 2] = -dxds[4 * k + 1];
      dsdx[4 * k + 3] = dxds[4 * k + 0];
    }
    TensorBoundaryInterp2D(interp.bM.data(), dsdx.data(), dsdxB.data(), N, 1, nEl);
    for (int e = 0; e < nEl; ++e)
      for (int k = 0; k < 4; ++k)
        for (int i = 0; i < P; ++i) {
          size_t b = i + P * (k + 4 * (size_t)e);
          double fac = (k == 1 || k == 2) ? std::copysign(1.0, JB[b]) : -std::copysign(1.0, JB[b]);
          int col = (k == 0 || k == 2) ? 1 : 0;  // South/North use dsdx(:,2); East/West dsdx(:,1)
          double a0 = dsdxB[4 * b + 0 + 2 * col], a1 = dsdxB[4 * b + 1 + 2 * col];
          double mag = std::sqrt(a0 * a0 + a1 * a1);
          nScale[b] = mag;
          nHat[2 * b + 0] = fac * a0 / mag;
          nHat[2 * b + 1] = fac * a1 / mag;
          for (int q = 0; q < 4; ++q) dsdxB[4 * b + q] = dsdxB[4 * b + q] * fac;
        }
  }

  // src/SELF_Geometry.f90:554-582
  double CovariantArcMin() const {
    int P = N + 1;
    double m = HUGE_VAL;
    for (size_t k = 0; k < (size_t)P * P * nEl; ++k) {
      double d11 = dxds[4 * k + 0], d21 = dxds[4 * k + 1], d12 = dxds[4 * k + 2], d22 = dxds[4 * k + 3];
      double dx = std::sqrt(d11 * d11 + d12 * d12);
      double dy = std::sqrt(d21 * d21 + d22 * d22);
      double ds = 2.0 * std::min(dx, dy) / ((double)N * (double)N);
      m = std::min(m, ds);
    }
    return m;
  }
};

// -------------------------------------------------------------------- models
// Williamson low-storage RK3, src/SELF_Model.f90:26-29
static const double rk3_a[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
static const double rk3_b[3] = {0.0, 1.0 / 3.0, 3.0 / 4.0};
static const double rk3_g[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};

enum Kind { LSW = 1, SW = 2, CIG = 3 };

struct Field {  // interior + boundary + extBoundary of a MappedScalar2D
  Vec in, b, ext;
};

struct Model {
  Kind kind;
  int N, P, nVar, nEl;
  Lagrange interp;
  std::vector<int> sideInfo;
  const SEMQuad* geo = nullptr;
  SEMQuad geoOwn;
  double g = 1.0, fCoriConst = 0.0;                     // LSW / SW
  double Cp = 1.4, Cv = 1.0, R = 1.0, gamma = 1.4;      // CIG
  Field sol, src, fdiv, dSdt, workSol;
  Vec flux, fluxBN;  // vector interior, boundaryNormal (P,nVar,4,nEl)
  // LSW
  Field Hb, fCori;
  // SW
  Field topo;
  Vec gradTopo, velIn, velB, velExt;
  // CIG
  Field prim, diag, prescSol, prescPrim, prescDiag, env;
  Vec envGrad;
  // artificial-viscosity closure (CIG): 0 off, 1 modal-decay indicator, 2 element viscosity given
  int closure = 0;
  bool avHeld = false;  // inside an RK step after its first stage: the step's element viscosity is kept
  double avC = 1.0, avS0 = 0.0, avKappa = 1.0;
  Vec modalT, avNu, avAct, avH, avAvg, avGrad, avGB, avGExt;

  size_t nIn(int nv) const { return (size_t)P * P * nv * nEl; }
  size_t nB(int nv) const { return (size_t)P * nv * 4 * nEl; }
  void alloc(Field& f, int nv) {
    f.in.assign(nIn(nv), 0.0);
    f.b.assign(nB(nv), 0.0);
    f.ext.assign(nB(nv), 0.0);
  }

  void init(Kind k, int N_, int quad, int nEl_, const int* si, const SEMQuad* g_) {
    kind = k;
    N = N_;
    P = N + 1;
    nEl = nEl_;
    nVar = (k == CIG) ? 4 : 3;
    interp.init(N, quad, N, UNIFORM);
    sideInfo.assign(si, si + 20 * (size_t)nEl);
    geo = g_;
    for (Field* f : {&sol, &src, &fdiv, &dSdt, &workSol}) alloc(*f, nVar);
    flux.assign(2 * nIn(nVar), 0.0);
    fluxBN.assign(nB(nVar), 0.0);
    if (k == LSW) {
      alloc(Hb, 1);
      alloc(fCori, 1);
    } else if (k == SW) {
      alloc(topo, 1);
      gradTopo.assign(2 * nIn(1), 0.0);
      velIn.assign(2 * nIn(1), 0.0);
      velB.assign(2 * nB(1), 0.0);
      velExt.assign(2 * nB(1), 0.0);
    } else {
      for (Field* f : {&prim, &diag, &prescSol, &prescPrim, &prescDiag}) alloc(*f, 4);
      alloc(env, 2);
      envGrad.assign(2 * nIn(2), 0.0);
    }
  }

  // --- LinearShallowWater (src/models/SELF_LinearShallowWater.f90)
  void lswBC() {  // :298-355
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s)
        for (int i = 0; i < P; ++i) {
          const int* si = &sideInfo[5 * (s + 4 * (size_t)e)];
          int bcid = si[4], e2 = si[2];
          if (e2 != 0) continue;
          if (bcid == BC_NONORMALFLOW) {
            size_t b = i + P * (s + 4 * (size_t)e);
            double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1];
            double u = sol.b[SCB(i, 0, s, e)], v = sol.b[SCB(i, 1, s, e)];
            sol.ext[SCB(i, 0, s, e)] = (n2 * n2 - n1 * n1) * u - 2.0 * n1 * n2 * v;
            sol.ext[SCB(i, 1, s, e)] = (n1 * n1 - n2 * n2) * v - 2.0 * n1 * n2 * u;
            sol.ext[SCB(i, 2, s, e)] = sol.b[SCB(i, 2, s, e)];
          } else {  // RADIATION and default
            sol.ext[SCB(i, 0, s, e)] = 0.0;
            sol.ext[SCB(i, 1, s, e)] = 0.0;
            sol.ext[SCB(i, 2, s, e)] = 0.0;
          }
        }
  }
  void lswSource() {  // :413-446
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double f = fCori.in[i + P * (j + P * (size_t)e)];
          src.in[SC(i, j, 0, e)] = f * sol.in[SC(i, j, 1, e)];
          src.in[SC(i, j, 1, e)] = -f * sol.in[SC(i, j, 0, e)];
          src.in[SC(i, j, 2, e)] = 0.0;
        }
  }
  void lswFlux() {  // :448-498
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double H = Hb.in[i + P * (j + P * (size_t)e)];
          flux[VE(0, i, j, 0, e)] = g * sol.in[SC(i, j, 2, e)];
          flux[VE(1, i, j, 0, e)] = 0.0;
          flux[VE(0, i, j, 1, e)] = 0.0;
          flux[VE(1, i, j, 1, e)] = g * sol.in[SC(i, j, 2, e)];
          flux[VE(0, i, j, 2, e)] = H * sol.in[SC(i, j, 0, e)];
          flux[VE(1, i, j, 2, e)] = H * sol.in[SC(i, j, 1, e)];
        }
  }
  void lswRiemann() {  // :500-557
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s)
        for (int i = 0; i < P; ++i) {
          size_t b = i + P * (s + 4 * (size_t)e);
          double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1], nmag = geo->nScale[b];
          double c = std::sqrt(g * Hb.b[b]);
          double unL = sol.b[SCB(i, 0, s, e)] * n1 + sol.b[SCB(i, 1, s, e)] * n2;
          double unR = sol.ext[SCB(i, 0, s, e)] * n1 + sol.ext[SCB(i, 1, s, e)] * n2;
          double etaL = sol.b[SCB(i, 2, s, e)], etaR = sol.ext[SCB(i, 2, s, e)];
          double wL = 0.5 * (unL / g + etaL / c);
          double wR = 0.5 * (unR / g - etaR / c);
          fluxBN[SCB(i, 0, s, e)] = g * c * (wL - wR) * n1 * nmag;
          fluxBN[SCB(i, 1, s, e)] = g * c * (wL - wR) * n2 * nmag;
          fluxBN[SCB(i, 2, s, e)] = c * c * (wL + wR) * nmag;
        }
  }

  // --- ShallowWater (src/models/SELF_ShallowWater.f90)
  void swPreTendency() {  // :190-239 (velocity traces come from the PREVIOUS solution%boundary)
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double H = sol.in[SC(i, j, 2, e)];
          size_t k = i + P * (j + P * (size_t)e);
          velIn[2 * k + 0] = sol.in[SC(i, j, 0, e)] / H;
          velIn[2 * k + 1] = sol.in[SC(i, j, 1, e)] / H;
        }
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s)
        for (int i = 0; i < P; ++i) {
          double H = sol.b[SCB(i, 2, s, e)];
          size_t b = i + P * (s + 4 * (size_t)e);
          velB[2 * b + 0] = sol.b[SCB(i, 0, s, e)] / H;
          velB[2 * b + 1] = sol.b[SCB(i, 1, s, e)] / H;
        }
    SideExchangeVector(velExt.data(), velB.data(), sideInfo.data(), N, 1, nEl);
  }
  void swBC() {  // :284-343
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s)
        for (int i = 0; i < P; ++i) {
          const int* si = &sideInfo[5 * (s + 4 * (size_t)e)];
          int bcid = si[4], e2 = si[2];
          if (e2 != 0) continue;
          size_t b = i + P * (s + 4 * (size_t)e);
          if (bcid == BC_NONORMALFLOW) {
            double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1];
            double u = sol.b[SCB(i, 0, s, e)], v = sol.b[SCB(i, 1, s, e)];
            sol.ext[SCB(i, 0, s, e)] = (n2 * n2 - n1 * n1) * u - 2.0 * n1 * n2 * v;
            sol.ext[SCB(i, 1, s, e)] = (n1 * n1 - n2 * n2) * v - 2.0 * n1 * n2 * u;
            sol.ext[SCB(i, 2, s, e)] = sol.b[SCB(i, 2, s, e)];
          } else {  // RADIATION and default
            sol.ext[SCB(i, 0, s, e)] = 0.0;
            sol.ext[SCB(i, 1, s, e)] = 0.0;
            sol.ext[SCB(i, 2, s, e)] = topo.b[b];
          }
        }
  }
  void swSource() {  // :345-384
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          size_t k = i + P * (j + P * (size_t)e);
          src.in[SC(i, j, 0, e)] = -fCoriConst * sol.in[SC(i, j, 1, e)] +
                                   g * sol.in[SC(i, j, 2, e)] * gradTopo[2 * k + 0];
          src.in[SC(i, j, 1, e)] = fCoriConst * sol.in[SC(i, j, 0, e)] +
                                   g * sol.in[SC(i, j, 2, e)] * gradTopo[2 * k + 1];
          src.in[SC(i, j, 2, e)] = 0.0;
        }
  }
  void swFlux() {  // :386-449
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          size_t k = i + P * (j + P * (size_t)e);
          double u = velIn[2 * k], v = velIn[2 * k + 1];
          double Hu = sol.in[SC(i, j, 0, e)], Hv = sol.in[SC(i, j, 1, e)], H = sol.in[SC(i, j, 2, e)];
          flux[VE(0, i, j, 0, e)] = u * Hu + 0.5 * g * H * H;
          flux[VE(1, i, j, 0, e)] = v * Hu;
          flux[VE(0, i, j, 1, e)] = u * Hv;
          flux[VE(1, i, j, 1, e)] = v * Hv + 0.5 * g * H * H;
          flux[VE(0, i, j, 2, e)] = Hu;
          flux[VE(1, i, j, 2, e)] = Hv;
        }
  }
  void swRiemann() {  // :451-529
    int nVar = 3;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s)
        for (int i = 0; i < P; ++i) {
          size_t b = i + P * (s + 4 * (size_t)e);
          double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1], nmag = geo->nScale[b];
          double unL = velB[2 * b] * n1 + velB[2 * b + 1] * n2;
          double unR = velExt[2 * b] * n1 + velExt[2 * b + 1] * n2;
          double cL = std::sqrt(g * sol.b[SCB(i, 2, s, e)]);
          double cR = std::sqrt(g * sol.ext[SCB(i, 2, s, e)]);
          double HuL = sol.b[SCB(i, 0, s, e)], HuR = sol.ext[SCB(i, 0, s, e)];
          double HvL = sol.b[SCB(i, 1, s, e)], HvR = sol.ext[SCB(i, 1, s, e)];
          double HL = sol.b[SCB(i, 2, s, e)], HR = sol.ext[SCB(i, 2, s, e)];
          double fL1 = HuL * unL + g * HL * HL * 0.5 * n1;
          double fL2 = HvL * unL + g * HL * HL * 0.5 * n2;
          double fL3 = HuL * n1 + HvL * n2;
          double fR1 = HuR * unR + g * HR * HR * 0.5 * n1;
          double fR2 = HvR * unR + g * HR * HR * 0.5 * n2;
          double fR3 = HuR * n1 + HvR * n2;
          double alpha = std::max(std::max(std::fabs(unL + cL), std::fabs(unR + cR)),
                                  std::max(std::fabs(unL - cL), std::fabs(unR - cR)));
          fluxBN[SCB(i, 0, s, e)] = 0.5 * (fL1 + fR1 + alpha * (HuL - HuR)) * nmag;
          fluxBN[SCB(i, 1, s, e)] = 0.5 * (fL2 + fR2 + alpha * (HvL - HvR)) * nmag;
          fluxBN[SCB(i, 2, s, e)] = 0.5 * (fL3 + fR3 + alpha * (HL - HR)) * nmag;
        }
  }

  // --- CompressibleIdealGas2D (src/models/SELF_CompressibleIdealGas2D.f90)
  void cigPreTendency() {  // :955-982, CalculateDiagnostics :984-1127, C2P :1129-1170
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double rhoU = sol.in[SC(i, j, 0, e)], rhoV = sol.in[SC(i, j, 1, e)];
          double rho = sol.in[SC(i, j, 2, e)], rhoE = sol.in[SC(i, j, 3, e)];
          double u = rhoU / rho, v = rhoV / rho;
          double rhoKE = 0.5 * (rhoU * u + rhoV * v);
          double p = (gamma - 1.0) * (rhoE - rhoKE);
          diag.in[SC(i, j, 0, e)] = rhoKE;
          diag.in[SC(i, j, 1, e)] = rhoE + p;
          diag.in[SC(i, j, 2, e)] = std::sqrt(gamma * p / rho);
          diag.in[SC(i, j, 3, e)] = (2.0 / 3.0) * ((rhoE - rhoKE) / rho) / R;
          prim.in[SC(i, j, 0, e)] = u;
          prim.in[SC(i, j, 1, e)] = v;
          prim.in[SC(i, j, 2, e)] = rho;
          prim.in[SC(i, j, 3, e)] = p;
        }
    // Entropy variables (:1172-1215) are computed and exchanged by the
    // reference but never read by the tendency (H16); they are not formed here.
    ScalarBoundaryInterp2D(interp.bM.data(), prim.in.data(), prim.b.data(), N, 4, nEl);
    ScalarBoundaryInterp2D(interp.bM.data(), diag.in.data(), diag.b.data(), N, 4, nEl);
    SideExchangeScalar(prim.ext.data(), prim.b.data(), sideInfo.data(), N, 4, nEl);
    SideExchangeScalar(diag.ext.data(), diag.b.data(), sideInfo.data(), N, 4, nEl);
  }
  void cigBC() {  // :1217-1323
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s) {
        const int* si = &sideInfo[5 * (s + 4 * (size_t)e)];
        int bcid = si[4], e2 = si[2];
        if (e2 != 0) continue;
        if (bcid == BC_NONORMALFLOW) {
          for (int i = 0; i < P; ++i) {
            size_t b = i + P * (s + 4 * (size_t)e);
            double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1];
            double u = sol.b[SCB(i, 0, s, e)], v = sol.b[SCB(i, 1, s, e)];
            sol.ext[SCB(i, 0, s, e)] = (n2 * n2 - n1 * n1) * u - 2.0 * n1 * n2 * v;
            sol.ext[SCB(i, 1, s, e)] = (n1 * n1 - n2 * n2) * v - 2.0 * n1 * n2 * u;
            sol.ext[SCB(i, 2, s, e)] = sol.b[SCB(i, 2, s, e)];
            sol.ext[SCB(i, 3, s, e)] = sol.b[SCB(i, 3, s, e)];
            u = prim.b[SCB(i, 0, s, e)];
            v = prim.b[SCB(i, 1, s, e)];
            prim.ext[SCB(i, 0, s, e)] = (n2 * n2 - n1 * n1) * u - 2.0 * n1 * n2 * v;
            prim.ext[SCB(i, 1, s, e)] = (n1 * n1 - n2 * n2) * v - 2.0 * n1 * n2 * u;
            prim.ext[SCB(i, 2, s, e)] = prim.b[SCB(i, 2, s, e)];
            prim.ext[SCB(i, 3, s, e)] = prim.b[SCB(i, 3, s, e)];
            for (int d = 0; d < 4; ++d) diag.ext[SCB(i, d, s, e)] = diag.b[SCB(i, d, s, e)];
          }
        } else if (bcid == BC_PRESCRIBED || bcid == BC_RADIATION) {
          for (int i = 0; i < P; ++i)
            for (int v = 0; v < 4; ++v) {
              sol.ext[SCB(i, v, s, e)] = prescSol.b[SCB(i, v, s, e)];
              prim.ext[SCB(i, v, s, e)] = prescPrim.b[SCB(i, v, s, e)];
              diag.ext[SCB(i, v, s, e)] = prescDiag.b[SCB(i, v, s, e)];
            }
        }
      }
  }
  void cigSource() {  // :1325-1366
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double rhou = sol.in[SC(i, j, 0, e)], rhov = sol.in[SC(i, j, 1, e)];
          double rho = sol.in[SC(i, j, 2, e)];
          // environmentalsGradient is a 2-variable vector field; variable 1 is used.
          size_t gk = 2 * (i + P * (j + P * (2 * (size_t)e)));
          double gx = envGrad[gk + 0], gy = envGrad[gk + 1];
          double Cd = env.in[i + P * (j + P * (1 + 2 * (size_t)e))];
          src.in[SC(i, j, 0, e)] = -rho * gx - Cd * rhou;
          src.in[SC(i, j, 1, e)] = -rho * gy - Cd * rhov;
          src.in[SC(i, j, 2, e)] = 0.0;
          src.in[SC(i, j, 3, e)] = -rhou * gx - rhou * gy;
        }
  }
  void cigFlux() {  // :1368-1440
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double u = prim.in[SC(i, j, 0, e)], v = prim.in[SC(i, j, 1, e)], p = prim.in[SC(i, j, 3, e)];
          double rhoU = sol.in[SC(i, j, 0, e)], rhoV = sol.in[SC(i, j, 1, e)];
          double rhoH = diag.in[SC(i, j, 1, e)];
          flux[VE(0, i, j, 0, e)] = u * rhoU + p;
          flux[VE(1, i, j, 0, e)] = v * rhoU;
          flux[VE(0, i, j, 1, e)] = u * rhoV;
          flux[VE(1, i, j, 1, e)] = v * rhoV + p;
          flux[VE(0, i, j, 2, e)] = rhoU;
          flux[VE(1, i, j, 2, e)] = rhoV;
          flux[VE(0, i, j, 3, e)] = u * rhoH;
          flux[VE(1, i, j, 3, e)] = v * rhoH;
        }
  }
  void cigLLF() {  // :1455-1542
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s)
        for (int i = 0; i < P; ++i) {
          size_t b = i + P * (s + 4 * (size_t)e);
          double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1], nmag = geo->nScale[b];
          double unL = prim.b[SCB(i, 0, s, e)] * n1 + prim.b[SCB(i, 1, s, e)] * n2;
          double unR = prim.ext[SCB(i, 0, s, e)] * n1 + prim.ext[SCB(i, 1, s, e)] * n2;
          double fL[4], fR[4], jump[4];
          fL[0] = unL * sol.b[SCB(i, 0, s, e)] + prim.b[SCB(i, 3, s, e)] * n1;
          fL[1] = unL * sol.b[SCB(i, 1, s, e)] + prim.b[SCB(i, 3, s, e)] * n2;
          fL[2] = sol.b[SCB(i, 0, s, e)] * n1 + sol.b[SCB(i, 1, s, e)] * n2;
          fL[3] = unL * diag.b[SCB(i, 1, s, e)];
          fR[0] = unR * sol.ext[SCB(i, 0, s, e)] + prim.ext[SCB(i, 3, s, e)] * n1;
          fR[1] = unR * sol.ext[SCB(i, 1, s, e)] + prim.ext[SCB(i, 3, s, e)] * n2;
          fR[2] = sol.ext[SCB(i, 0, s, e)] * n1 + sol.ext[SCB(i, 1, s, e)] * n2;
          fR[3] = unR * diag.ext[SCB(i, 1, s, e)];
          for (int v = 0; v < 4; ++v) jump[v] = sol.b[SCB(i, v, s, e)] - sol.ext[SCB(i, v, s, e)];
          double cL = diag.b[SCB(i, 2, s, e)], cR = diag.ext[SCB(i, 2, s, e)];
          double alpha = std::max(std::fabs(unL), std::fabs(unR)) + std::max(std::fabs(cL), std::fabs(cR));
          for (int v = 0; v < 4; ++v) fluxBN[SCB(i, v, s, e)] = 0.5 * (fL[v] + fR[v] + alpha * jump[v]) * nmag;
        }
  }

  // --- artificial-viscosity closure (see the closure helpers above)
  void closureEnable(int mode, double c, double s0, double kappa) {
    closure = mode;
    avC = c;
    avS0 = s0;
    avKappa = kappa;
    modalT.assign((size_t)P * P, 0.0);
    ModalMatrix(N, interp.ctrl.data(), interp.qw.data(), modalT.data());
    if (avNu.size() != (size_t)nEl) avNu.assign(nEl, 0.0);
    avAct.assign(nEl, 0.0);
    avH.assign(nEl, 0.0);
    for (int e = 0; e < nEl; ++e) {  // h = sqrt(sum_ij w_i w_j J_ij)
      double area = 0.0;
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) area = area + interp.qw[i] * interp.qw[j] * geo->J[i + P * (j + P * (size_t)e)];
      avH[e] = std::sqrt(area);
    }
    avAvg.assign(nB(4), 0.0);
    avGrad.assign(2 * nIn(4), 0.0);
    avGB.assign(2 * nB(4), 0.0);
    avGExt.assign(2 * nB(4), 0.0);
  }
  // element viscosity from the modal-decay indicator of the density (closure 1)
  void cigClosureViscosity() {
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e) {
      double c[kOrcMaxP * kOrcMaxP];
      ModalCoefficients(modalT.data(), &sol.in[SC(0, 0, 2, e)], c, P);
      double a = ModalDecayActivation(c, P, avS0, avKappa);
      double lam = 0.0;
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double u = prim.in[SC(i, j, 0, e)], v = prim.in[SC(i, j, 1, e)];
          double w = std::sqrt(u * u + v * v) + diag.in[SC(i, j, 2, e)];
          if (w > lam) lam = w;
        }
      avAct[e] = a;
      avNu[e] = a * avC * avH[e] / (double)N * lam;
    }
  }
  // BR1 gradient of the conservative variables and the viscous traces nu grad q
  void cigClosureGradient() {
    int nVar = 4;
    BassiRebaySides(avAvg.data(), sol.b.data(), sol.ext.data(), N, 4, nEl);
    GradientBR(sol.in.data(), avAvg.data(), geo->dsdx.data(), geo->J.data(), geo->nHat.data(), geo->nScale.data(),
               avGrad.data(), interp.dgM.data(), interp.bM.data(), interp.qw.data(), N, 4, nEl);
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (size_t k = 0; k < 2 * (size_t)P * P * 4; ++k) avGrad[k + 2 * (size_t)P * P * 4 * e] *= avNu[e];
    VectorBoundaryInterp2D(interp.bM.data(), avGrad.data(), avGB.data(), N, 4, nEl);
    SideExchangeVector(avGExt.data(), avGB.data(), sideInfo.data(), N, 4, nEl);
  }
  // viscous contributions on the contravariant volume flux and on the face flux
  void cigClosureFluxes() {
    int nVar = 4;
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int v = 0; v < 4; ++v)
        for (int j = 0; j < P; ++j)
          for (int i = 0; i < P; ++i) {
            size_t a = 4 * (i + P * (j + P * (size_t)e));
            double gx = avGrad[VE(0, i, j, v, e)], gy = avGrad[VE(1, i, j, v, e)];
            double f1 = -(geo->dsdx[a + 0] * gx + geo->dsdx[a + 1] * gy);
            double f2 = -(geo->dsdx[a + 2] * gx + geo->dsdx[a + 3] * gy);
            flux[VE(0, i, j, v, e)] = flux[VE(0, i, j, v, e)] + f1;
            flux[VE(1, i, j, v, e)] = flux[VE(1, i, j, v, e)] + f2;
          }
    OMP_FOR
    for (int e = 0; e < nEl; ++e)
      for (int s = 0; s < 4; ++s) {
        if (sideInfo[5 * (s + 4 * (size_t)e) + 4] != 0) continue;  // no viscous flux through physical sides
        for (int v = 0; v < 4; ++v)
          for (int i = 0; i < P; ++i) {
            size_t b = i + P * (s + 4 * (size_t)e);
            double n1 = geo->nHat[2 * b], n2 = geo->nHat[2 * b + 1], nmag = geo->nScale[b];
            double in = avGB[VEB(0, i, v, s, e)] * n1 + avGB[VEB(1, i, v, s, e)] * n2;
            double ex = avGExt[VEB(0, i, v, s, e)] * n1 + avGExt[VEB(1, i, v, s, e)] * n2;
            fluxBN[SCB(i, v, s, e)] = fluxBN[SCB(i, v, s, e)] + -0.5 * (in + ex) * nmag;
          }
      }
  }

  // src/SELF_Model2D.f90:816-859
  void CalculateTendency() {
    if (kind == SW) swPreTendency();
    if (kind == CIG) cigPreTendency();
    ScalarBoundaryInterp2D(interp.bM.data(), sol.in.data(), sol.b.data(), N, nVar, nEl);
    SideExchangeScalar(sol.ext.data(), sol.b.data(), sideInfo.data(), N, nVar, nEl);
    if (kind == LSW) { lswBC(); lswSource(); lswRiemann(); lswFlux(); }
    if (kind == SW) { swBC(); swSource(); swRiemann(); swFlux(); }
    if (kind == CIG) { cigBC(); cigSource(); cigLLF(); cigFlux(); }
    if (kind == CIG && closure != 0) {
      if (closure == 1 && !avHeld) cigClosureViscosity();
      cigClosureGradient();
    }
    ContravariantProjection(flux.data(), geo->dsdx.data(), N, nVar, nEl);
    if (kind == CIG && closure != 0) cigClosureFluxes();
    VectorDGDivergence2D(interp.dgM.data(), interp.bM.data(), interp.qw.data(), flux.data(),
                         fluxBN.data(), fdiv.in.data(), N, nVar, nEl);
    JacobianWeightScalar(fdiv.in.data(), geo->J.data(), N, nVar, nEl);
    size_t n = nIn(nVar);
    OMP_FOR
    for (long long k = 0; k < (long long)n; ++k) dSdt.in[k] = src.in[k] - fdiv.in[k];
  }

  // src/SELF_Model2D.f90:710-752
  void UpdateGRK3(int m, double dt) {
    size_t n = nIn(nVar);
    OMP_FOR
    for (long long k = 0; k < (long long)n; ++k) {
      workSol.in[k] = rk3_a[m] * workSol.in[k] + dSdt.in[k];
      sol.in[k] = sol.in[k] + rk3_g[m] * dt * workSol.in[k];
    }
  }

  // src/SELF_Model.f90:704-732, stepped by count (H15)
  // The closure's element viscosity (closure 1) is formed at each step's
  // first stage and held over the step's other two (the engine's closure does
  // the same; not a reference routine).
  void RK3(int nSteps, double dt) {
    for (int s = 0; s < nSteps; ++s)
      for (int m = 0; m < 3; ++m) {
        avHeld = m > 0;
        CalculateTendency();
        UpdateGRK3(m, dt);
      }
    avHeld = false;
  }

  double Entropy() const {
    int nVar = this->nVar;
    double ent = 0.0;
    for (int e = 0; e < nEl; ++e)
      for (int j = 0; j < P; ++j)
        for (int i = 0; i < P; ++i) {
          double Jac = geo->J[i + P * (j + P * (size_t)e)];
          double wi = interp.qw[i], wj = interp.qw[j];
          if (kind == LSW) {  // src/models/SELF_LinearShallowWater.f90:171-216
            double u = sol.in[SC(i, j, 0, e)], v = sol.in[SC(i, j, 1, e)], eta = sol.in[SC(i, j, 2, e)];
            double H = Hb.in[i + P * (j + P * (size_t)e)];
            ent = ent + 0.5 * (H * (u * u + v * v) + g * eta * eta) * Jac * wi * wj;
          } else if (kind == SW) {  // src/models/SELF_ShallowWater.f90:149-188
            double Hu = sol.in[SC(i, j, 0, e)], Hv = sol.in[SC(i, j, 1, e)], H = sol.in[SC(i, j, 2, e)];
            double b = topo.in[i + P * (j + P * (size_t)e)];
            ent = ent + (0.5 * (Hu * Hu / H + Hv * Hv / H) + 0.5 * g * H * H - g * H * b) * Jac * wi * wj;
          } else {  // src/models/SELF_CompressibleIdealGas2D.f90:782-823
            double rho = sol.in[SC(i, j, 2, e)], p = prim.in[SC(i, j, 3, e)];
            ent = ent + rho * (std::log(p) - gamma * std::log(rho)) / (gamma - 1.0) * wi * wj * Jac;
          }
        }
    return ent;
  }
};

}  // namespace orc

// ===================================================================== C ABI
using namespace orc;

extern "C" {

int orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void orc_legendre_quadrature(int N, int type, double* x, double* w) {
  if (type == GAUSS) LegendreGauss(N, x, w);
  else if (type == GAUSS_LOBATTO) LegendreGaussLobatto(N, x, w);
  else ChebyshevQuad(N, type, x, w);
}

// Lagrange%Init outputs, Fortran layouts.
void orc_lagrange(int N, int ctrl, int M, int tgt, double* ctrlPts, double* tgtPts, double* bw,
                  double* qw, double* iM, double* dM, double* dgM, double* bM) {
  Lagrange L;
  L.init(N, ctrl, M, tgt);
  std::memcpy(ctrlPts, L.ctrl.data(), sizeof(double) * L.ctrl.size());
  std::memcpy(tgtPts, L.tgt.data(), sizeof(double) * L.tgt.size());
  std::memcpy(bw, L.bw.data(), sizeof(double) * L.bw.size());
  std::memcpy(qw, L.qw.data(), sizeof(double) * L.qw.size());
  std::memcpy(iM, L.iM.data(), sizeof(double) * L.iM.size());
  std::memcpy(dM, L.dM.data(), sizeof(double) * L.dM.size());
  std::memcpy(dgM, L.dgM.data(), sizeof(double) * L.dgM.size());
  std::memcpy(bM, L.bM.data(), sizeof(double) * L.bM.size());
}

void orc_scalar_boundary_interp_2d(const double* bM, const double* f, double* fb, int N, int nVar, int nEl) {
  ScalarBoundaryInterp2D(bM, f, fb, N, nVar, nEl);
}
void orc_vector_boundary_interp_2d(const double* bM, const double* f, double* fb, int N, int nVar, int nEl) {
  VectorBoundaryInterp2D(bM, f, fb, N, nVar, nEl);
}
void orc_tensor_boundary_interp_2d(const double* bM, const double* f, double* fb, int N, int nVar, int nEl) {
  TensorBoundaryInterp2D(bM, f, fb, N, nVar, nEl);
}
void orc_scalar_grid_interp_2d(const double* iM, const double* f, double* fo, int N, int M, int nVar, int nEl) {
  ScalarGridInterp2D(iM, f, fo, N, M, nVar, nEl);
}
void orc_vector_grid_interp_2d(const double* iM, const double* f, double* fo, int N, int M, int nVar, int nEl) {
  VectorGridInterp2D(iM, f, fo, N, M, nVar, nEl);
}
void orc_vector_gradient_2d(const double* dM, const double* f, double* gf, int N, int nVar, int nEl) {
  VectorGradient2D(dM, f, gf, N, nVar, nEl);
}
void orc_vector_dg_divergence_2d(const double* dgM, const double* bM, const double* qw, const double* f,
                                 const double* bf, double* df, int N, int nVar, int nEl) {
  VectorDGDivergence2D(dgM, bM, qw, f, bf, df, N, nVar, nEl);
}
void orc_jacobian_weight_2d(double* f, const double* J, int N, int nVar, int nEl) {
  JacobianWeightScalar(f, J, N, nVar, nEl);
}
void orc_contravariant_projection_2d(double* f, const double* dsdx, int N, int nVar, int nEl) {
  ContravariantProjection(f, dsdx, N, nVar, nEl);
}
void orc_side_exchange_scalar_2d(double* ext, const double* bnd, const int* sideInfo, int N, int nVar, int nEl) {
  SideExchangeScalar(ext, bnd, sideInfo, N, nVar, nEl);
}
void orc_side_exchange_vector_2d(double* ext, const double* bnd, const int* sideInfo, int N, int nVar, int nEl) {
  SideExchangeVector(ext, bnd, sideInfo, N, nVar, nEl);
}
void orc_bassi_rebay_sides_2d(double* avg, const double* bnd, const double* ext, int N, int nVar, int nEl) {
  BassiRebaySides(avg, bnd, ext, N, nVar, nEl);
}
void orc_gradient_sf_2d(const double* f, const double* dsdx, const double* J, double* gradF, const double* dM,
                        int N, int nVar, int nEl) {
  GradientSF(f, dsdx, J, gradF, dM, N, nVar, nEl);
}
void orc_gradient_br_2d(const double* f, const double* avgB, const double* dsdx, const double* J,
                        const double* nHat, const double* nScale, double* gradF, const double* dgM,
                        const double* bM, const double* qw, int N, int nVar, int nEl) {
  GradientBR(f, avgB, dsdx, J, nHat, nScale, gradF, dgM, bM, qw, N, nVar, nEl);
}
void orc_determinant_2d(const double* t, double* det, int N, int nVar, int nEl) {
  Determinant2D(t, det, N, nVar, nEl);
}

// Structured mesh: nodeCoords (2,2,2,nEl), globalNodeIDs (2,2,nEl), sideInfo (5,4,nEl).
void orc_mesh_structured(int nx, int ny, double x0, double x1, double y0, double y1, int perX, int perY,
                         double amp, int bcid, const int* rot, double* nodeCoords, int* globalNodeIDs,
                         int* sideInfo) {
  Mesh2D m;
  m.Structured(nx, ny, x0, x1, y0, y1, perX, perY, amp, bcid, rot);
  std::memcpy(nodeCoords, m.nodeCoords.data(), sizeof(double) * m.nodeCoords.size());
  std::memcpy(globalNodeIDs, m.globalNodeIDs.data(), sizeof(int) * m.globalNodeIDs.size());
  std::memcpy(sideInfo, m.sideInfo.data(), sizeof(int) * m.sideInfo.size());
}

// SEMQuad%GenerateFromMesh for an nGeo = 1 mesh.  All outputs caller-allocated.
double orc_geometry(int N, int quad, int nEl, const double* nodeCoords, double* x, double* xB, double* dxds,
                    double* dxdsB, double* dsdx, double* dsdxB, double* J, double* JB, double* nHat,
                    double* nScale) {
  Lagrange L;
  L.init(N, quad, N, UNIFORM);
  Mesh2D m;
  m.nElem = nEl;
  m.nGeo = 1;
  m.nodeCoords.assign(nodeCoords, nodeCoords + 8 * (size_t)nEl);
  SEMQuad G;
  G.Generate(L, m);
  auto cp = [](double* d, const Vec& s) { std::memcpy(d, s.data(), sizeof(double) * s.size()); };
  cp(x, G.x);
  cp(xB, G.xB);
  cp(dxds, G.dxds);
  cp(dxdsB, G.dxdsB);
  cp(dsdx, G.dsdx);
  cp(dsdxB, G.dsdxB);
  cp(J, G.J);
  cp(JB, G.JB);
  cp(nHat, G.nHat);
  cp(nScale, G.nScale);
  return G.CovariantArcMin();
}

// ---- model handle
struct OrcModel {
  Model m;
  SEMQuad geo;
};

void* orc_model_create(int kind, int N, int quad, int nEl, const int* sideInfo, const double* nodeCoords) {
  OrcModel* h = new OrcModel();
  Lagrange L;
  L.init(N, quad, N, UNIFORM);
  Mesh2D mesh;
  mesh.nElem = nEl;
  mesh.nGeo = 1;
  mesh.nodeCoords.assign(nodeCoords, nodeCoords + 8 * (size_t)nEl);
  h->geo.Generate(L, mesh);
  h->m.init((Kind)kind, N, quad, nEl, sideInfo, &h->geo);
  return h;
}

void orc_model_free(void* p) { delete (OrcModel*)p; }

void orc_model_set_params(void* p, double g, double fCori, double Cp, double Cv, double R) {
  Model& m = ((OrcModel*)p)->m;
  m.g = g;
  m.fCoriConst = fCori;
  m.Cp = Cp;
  m.Cv = Cv;
  m.gamma = Cp / Cv;  // SetCp/SetCv, src/models/SELF_CompressibleIdealGas2D.f90:745-770
  m.R = R;
}

static Vec* field_ptr(Model& m, const std::string& n) {
  if (n == "solution") return &m.sol.in;
  if (n == "solution.boundary") return &m.sol.b;
  if (n == "solution.extBoundary") return &m.sol.ext;
  if (n == "dSdt") return &m.dSdt.in;
  if (n == "source") return &m.src.in;
  if (n == "fluxDivergence") return &m.fdiv.in;
  if (n == "workSol") return &m.workSol.in;
  if (n == "flux") return &m.flux;
  if (n == "flux.boundaryNormal") return &m.fluxBN;
  if (n == "H") return &m.Hb.in;
  if (n == "H.boundary") return &m.Hb.b;
  if (n == "fCori") return &m.fCori.in;
  if (n == "topography") return &m.topo.in;
  if (n == "topography.boundary") return &m.topo.b;
  if (n == "gradTopography") return &m.gradTopo;
  if (n == "velocity") return &m.velIn;
  if (n == "velocity.boundary") return &m.velB;
  if (n == "velocity.extBoundary") return &m.velExt;
  if (n == "primitive") return &m.prim.in;
  if (n == "primitive.boundary") return &m.prim.b;
  if (n == "primitive.extBoundary") return &m.prim.ext;
  if (n == "diagnostics") return &m.diag.in;
  if (n == "diagnostics.boundary") return &m.diag.b;
  if (n == "diagnostics.extBoundary") return &m.diag.ext;
  if (n == "environmentals") return &m.env.in;
  if (n == "environmentalsGradient") return &m.envGrad;
  if (n == "prescribedSolution.boundary") return &m.prescSol.b;
  if (n == "avNu") return m.avNu.empty() ? nullptr : &m.avNu;
  if (n == "avActivation") return m.avAct.empty() ? nullptr : &m.avAct;
  if (n == "avH") return m.avH.empty() ? nullptr : &m.avH;
  if (n == "avGradient") return m.avGrad.empty() ? nullptr : &m.avGrad;
  if (n == "avGradient.boundary") return m.avGB.empty() ? nullptr : &m.avGB;
  return nullptr;
}

// Copies `data` into the named field and applies the reference's follow-up for
// that setter: SetSolution -> BoundaryInterp (src/SELF_Model2D.f90:247-266);
// SetBathymetry -> BoundaryInterp (LSW :284-296); SetTopography ->
// BoundaryInterp + GradientSF (SW :241-282); SetGravity -> GradientSF (CIG
// :604-629); "prescribed" copies the current solution/primitive/diagnostics
// (SetPrescribedSolutionFromSolution, CIG :694-743).
int orc_model_set(void* p, const char* name, const double* data) {
  OrcModel* h = (OrcModel*)p;
  Model& m = h->m;
  std::string n(name);
  int P = m.P, N = m.N, nEl = m.nEl;
  if (n == "prescribed") {
    m.cigPreTendency();
    m.prescSol.in = m.sol.in;
    m.prescPrim.in = m.prim.in;
    m.prescDiag.in = m.diag.in;
    ScalarBoundaryInterp2D(m.interp.bM.data(), m.prescSol.in.data(), m.prescSol.b.data(), N, 4, nEl);
    ScalarBoundaryInterp2D(m.interp.bM.data(), m.prescPrim.in.data(), m.prescPrim.b.data(), N, 4, nEl);
    ScalarBoundaryInterp2D(m.interp.bM.data(), m.prescDiag.in.data(), m.prescDiag.b.data(), N, 4, nEl);
    return 0;
  }
  if (n == "gravityPotential") {
    for (int e = 0; e < nEl; ++e)
      for (int k = 0; k < P * P; ++k) m.env.in[k + P * P * (0 + 2 * (size_t)e)] = data[k + P * P * (size_t)e];
    GradientSF(m.env.in.data(), h->geo.dsdx.data(), h->geo.J.data(), m.envGrad.data(), m.interp.dM.data(), N, 2,
               nEl);
    return 0;
  }
  if (n == "drag") {
    for (int e = 0; e < nEl; ++e)
      for (int k = 0; k < P * P; ++k) m.env.in[k + P * P * (1 + 2 * (size_t)e)] = data[k + P * P * (size_t)e];
    return 0;
  }
  Vec* f = field_ptr(m, n);
  if (!f) return -1;
  std::memcpy(f->data(), data, sizeof(double) * f->size());
  if (n == "solution")
    ScalarBoundaryInterp2D(m.interp.bM.data(), m.sol.in.data(), m.sol.b.data(), N, m.nVar, nEl);
  if (n == "H") ScalarBoundaryInterp2D(m.interp.bM.data(), m.Hb.in.data(), m.Hb.b.data(), N, 1, nEl);
  if (n == "topography") {
    ScalarBoundaryInterp2D(m.interp.bM.data(), m.topo.in.data(), m.topo.b.data(), N, 1, nEl);
    GradientSF(m.topo.in.data(), h->geo.dsdx.data(), h->geo.J.data(), m.gradTopo.data(), m.interp.dM.data(), N,
               1, nEl);
  }
  return 0;
}

long long orc_model_field_size(void* p, const char* name) {
  OrcModel* h = (OrcModel*)p;
  std::string n(name);
  if (n.rfind("geometry.", 0) == 0) {
    SEMQuad& G = h->geo;
    if (n == "geometry.x") return G.x.size();
    if (n == "geometry.dsdx") return G.dsdx.size();
    if (n == "geometry.J") return G.J.size();
    if (n == "geometry.nHat") return G.nHat.size();
    if (n == "geometry.nScale") return G.nScale.size();
    if (n == "geometry.dxds") return G.dxds.size();
    return -1;
  }
  Vec* f = field_ptr(h->m, n);
  return f ? (long long)f->size() : -1;
}

int orc_model_get(void* p, const char* name, double* out) {
  OrcModel* h = (OrcModel*)p;
  std::string n(name);
  const Vec* f = nullptr;
  if (n == "geometry.x") f = &h->geo.x;
  else if (n == "geometry.dsdx") f = &h->geo.dsdx;
  else if (n == "geometry.J") f = &h->geo.J;
  else if (n == "geometry.nHat") f = &h->geo.nHat;
  else if (n == "geometry.nScale") f = &h->geo.nScale;
  else if (n == "geometry.dxds") f = &h->geo.dxds;
  else f = field_ptr(h->m, n);
  if (!f) return -1;
  std::memcpy(out, f->data(), sizeof(double) * f->size());
  return 0;
}

// closure 0 off, 1 modal-decay indicator, 2 element viscosity set through "avNu"
int orc_model_set_closure(void* p, int closure, double c, double s0, double kappa) {
  Model& m = ((OrcModel*)p)->m;
  if (m.kind != CIG || closure < 0 || closure > 2) return -1;
  m.closureEnable(closure, c, s0, kappa);
  return 0;
}

void orc_modal_matrix(int N, int quad, double* T) {
  Lagrange L;
  L.init(N, quad, N, UNIFORM);
  ModalMatrix(N, L.ctrl.data(), L.qw.data(), T);
}

// Per element of a (P,P,4,nEl) CIG state: modal-decay activation of the density
// and the 36 closure features (density, then total energy) in feat(36, nEl).
void orc_closure_features(const double* T, const double* q, int N, int nEl, double s0, double kappa, double* act,
                          double* feat) {
  int P = N + 1;
  OMP_FOR
  for (int e = 0; e < nEl; ++e) {
    double c[kOrcMaxP * kOrcMaxP];
    ModalCoefficients(T, q + (size_t)P * P * (2 + 4 * (size_t)e), c, P);
    if (act) act[e] = ModalDecayActivation(c, P, s0, kappa);
    if (feat) {
      ModalFeatures(c, P, feat + 36 * (size_t)e);
      ModalCoefficients(T, q + (size_t)P * P * (3 + 4 * (size_t)e), c, P);
      ModalFeatures(c, P, feat + 36 * (size_t)e + 18);
    }
  }
}

void orc_model_tendency(void* p) { ((OrcModel*)p)->m.CalculateTendency(); }
void orc_model_rk3(void* p, int nSteps, double dt) { ((OrcModel*)p)->m.RK3(nSteps, dt); }
double orc_model_entropy(void* p) {
  OrcModel* h = (OrcModel*)p;
  if (h->m.kind == CIG) h->m.cigPreTendency();
  return h->m.Entropy();
}
double orc_model_arcmin(void* p) { return ((OrcModel*)p)->geo.CovariantArcMin(); }

}  // extern "C"
