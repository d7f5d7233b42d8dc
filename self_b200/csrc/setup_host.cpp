// Host-side set-up for the engine: 1-D quadrature, the Lagrange operator
// matrices, and a structured quadrilateral mesh with SELF's sideInfo
// connectivity.  These are the inputs of the tendency path; they are small,
// built once, and reproduced here bit-for-bit against the reference's
// construction so that the device path sees the same operators:
//
//   * Legendre-Gauss / Gauss-Lobatto nodes by Newton iteration with the
//     reference's initial guess, exit test and mirrored fill
//     (src/SELF_Quadrature.f90:201-335).  At N = 3 this yields the Gauss nodes
//     in a mirrored but non-monotonic order; the order is kept because every
//     operator and the side flip (x_{N-i} = -x_i) stay consistent with it.
//   * barycentric weights, interpolation, derivative (strong and weak) and
//     boundary matrices built in double (src/SELF_Lagrange.f90:2542-2774).
//   * mesh corner/side conventions of src/SELF_Mesh.f90:30-90 with the flip
//     recomputed from shared corner ids as in RecalculateFlip_Mesh2D
//     (src/SELF_Mesh.f90:1018-1174).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "selfgpu_internal.h"

namespace selfgpu {

static thread_local std::string g_last_error;

int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
const char* last_error() { return g_last_error.c_str(); }

namespace {

const double kPi = 4.0 * std::atan(1.0);

// Legendre polynomial L_n and derivative by the three-term recurrence.
void legendre(int n, double x, double& l, double& dl) {
  if (n == 0) { l = 1.0; dl = 0.0; return; }
  if (n == 1) { l = x; dl = 1.0; return; }
  double l2 = 1.0, l1 = x, d2 = 0.0, d1 = 1.0;
  for (int k = 2; k <= n; ++k) {
    double dk = (double)k;
    l = ((2.0 * dk - 1.0) * x * l1 - (dk - 1.0) * l2) / dk;
    dl = d2 + (2.0 * dk - 1.0) * l1;
    l2 = l1; l1 = l; d2 = d1; d1 = dl;
  }
}

// q = L_{n+1} - L_{n-1}, its derivative, and L_n (Lobatto node function).
void lobatto_q(int n, double x, double& q, double& qp, double& ln) {
  double l2 = 1.0, l1 = x, d2 = 0.0, d1 = 1.0, dln = 0.0;
  ln = 0.0;
  for (int k = 2; k <= n; ++k) {
    double dk = (double)k;
    ln = (2.0 * k - 1.0) / dk * x * l1 - (dk - 1.0) / dk * l2;
    dln = d2 + (2.0 * dk - 1.0) * l1;
    l2 = l1; l1 = ln; d2 = d1; d1 = dln;
  }
  double dk = (double)(n + 1);
  double ln1 = (2.0 * (n + 1) - 1.0) / dk * x * ln - (dk - 1.0) / dk * l2;
  double dln1 = d2 + (2.0 * dk - 1.0) * l1;
  q = ln1 - l2;
  qp = dln1 - d2;
}

void gauss(int N, double* x, double* w) {
  std::vector<double> xs(N + 1, 0.0), ws(N + 1, 0.0);
  if (N == 0) {
    ws[0] = 2.0;
  } else if (N == 1) {
    // The reference reads its zero-initialised output for the mirrored node.
    xs[0] = -std::sqrt(1.0 / 3.0);
    ws[0] = 1.0;
    xs[1] = -0.0;
  } else {
    for (int j = 0; j <= (N + 1) / 2; ++j) {
      double xj = -std::cos((2.0 * j + 1.0) * kPi / (2.0 * N + 1.0));
      double l, dl;
      for (int it = 0; it < 500; ++it) {
        legendre(N + 1, xj, l, dl);
        double d = -l / dl;
        xj = xj + d;
        if (std::fabs(d) <= DBL_EPSILON * xj) break;
      }
      legendre(N + 1, xj, l, dl);
      xs[j] = xj;
      ws[j] = 2.0 / ((1.0 - xj * xj) * dl * dl);
      ws[N - j] = ws[j];
      xs[N - j] = -xs[j];
    }
  }
  if (N % 2 == 0) {
    double l, dl;
    legendre(N + 1, 0.0, l, dl);
    xs[N / 2] = 0.0;
    ws[N / 2] = 2.0 / (dl * dl);
  }
  std::copy(xs.begin(), xs.end(), x);
  std::copy(ws.begin(), ws.end(), w);
}

void gauss_lobatto(int N, double* x, double* w) {
  std::vector<double> xs(N + 1, 0.0), ws(N + 1, 0.0);
  double dN = (double)N;
  if (N == 1) {
    xs[0] = -1.0; ws[0] = 1.0; xs[1] = 1.0; ws[1] = 1.0;
  } else {
    xs[0] = -1.0;
    ws[0] = 2.0 / (dN * (dN + 1.0));
    xs[N] = 1.0;
    ws[N] = ws[0];
    for (int j = 1; j <= (N + 1) / 2 - 1; ++j) {
      double dj = (double)j;
      double xj = -std::cos((dj + 0.25) * kPi / dN - 3.0 / (8.0 * dN * kPi * (dj + 0.25)));
      double q, qp, ln;
      for (int it = 0; it < 500; ++it) {
        lobatto_q(N, xj, q, qp, ln);
        double d = -q / qp;
        xj = xj + d;
        if (std::fabs(d) <= DBL_EPSILON * xj) break;
      }
      lobatto_q(N, xj, q, qp, ln);
      xs[j] = xj;
      ws[j] = 2.0 / (dN * (dN + 1.0) * ln * ln);
      ws[N - j] = ws[j];
      xs[N - j] = -xs[j];
    }
  }
  if (N % 2 == 0) {
    double q, qp, ln;
    lobatto_q(N, 0.0, q, qp, ln);
    xs[N / 2] = 0.0;
    ws[N / 2] = 2.0 / (dN * (dN + 1.0) * ln * ln);
  }
  std::copy(xs.begin(), xs.end(), x);
  std::copy(ws.begin(), ws.end(), w);
}

bool almost_equal(double a, double b) {
  double d = std::fabs(a - b);
  if (a == 0.0 || b == 0.0) return d <= DBL_EPSILON;
  return d <= DBL_EPSILON * std::fabs(a) || d <= DBL_EPSILON * std::fabs(b);
}

void uniform(int n, double* x) {
  double dx = 2.0 / (double)n;
  for (int i = 0; i <= n; ++i) x[i] = -1.0 + dx * (double)i;
}

// Lagrange basis at s from barycentric weights; exact unit vector on a node.
void basis_at(int N, const double* ctrl, const double* bw, double s, double* out) {
  bool hit = false;
  for (int j = 0; j <= N; ++j) {
    out[j] = 0.0;
    if (almost_equal(s, ctrl[j])) { out[j] = 1.0; hit = true; }
  }
  if (hit) return;
  double sum = 0.0;
  for (int j = 0; j <= N; ++j) {
    out[j] = bw[j] / (s - ctrl[j]);
    sum = sum + out[j];
  }
  for (int j = 0; j <= N; ++j) out[j] = out[j] / sum;
}

}  // namespace

void legendre_quadrature(int N, int type, double* x, double* w) {
  if (type == SELFGPU_GAUSS_LOBATTO) gauss_lobatto(N, x, w);
  else gauss(N, x, w);
}

int lagrange_init(int N, int ctrlType, int M, int tgtType, double* ctrl, double* tgt, double* bw, double* qw,
                  double* iM, double* dM, double* dgM, double* bM) {
  if (N < 1 || N > SELFGPU_MAX_N || M < 0) return set_error(SELFGPU_ERR_ARG, "lagrange_init: bad degree");
  const int P = N + 1;
  if (ctrlType == SELFGPU_GAUSS || ctrlType == SELFGPU_GAUSS_LOBATTO) {
    legendre_quadrature(N, ctrlType, ctrl, qw);
  } else if (ctrlType == SELFGPU_UNIFORM) {
    uniform(N, ctrl);
    for (int i = 0; i < P; ++i) qw[i] = 2.0 / (double)N;
  } else {
    return set_error(SELFGPU_ERR_ARG, "lagrange_init: unsupported control node type");
  }
  std::vector<double> tq(M + 1);
  if (tgtType == SELFGPU_GAUSS || tgtType == SELFGPU_GAUSS_LOBATTO) legendre_quadrature(M, tgtType, tgt, tq.data());
  else uniform(M, tgt);
  // barycentric weights
  std::vector<double> b(P, 1.0);
  for (int j = 1; j <= N; ++j)
    for (int i = 0; i < j; ++i) {
      b[i] = b[i] * (ctrl[i] - ctrl[j]);
      b[j] = b[j] * (ctrl[j] - ctrl[i]);
    }
  for (int j = 0; j < P; ++j) bw[j] = 1.0 / b[j];
  // interpolation matrix, stored iM[ii + P*m]
  std::vector<double> row(P);
  for (int m = 0; m <= M; ++m) {
    basis_at(N, ctrl, bw, tgt[m], row.data());
    for (int ii = 0; ii < P; ++ii) iM[ii + (size_t)P * m] = row[ii];
  }
  // derivative matrices: D(r,c) = b_c / (b_r (x_r - x_c)), D(r,r) = -sum;
  // weak form G(r,c) = -D(c,r) w_c / w_r.  Stored transposed: dM[c + P*r] = D(r,c).
  std::vector<double> D((size_t)P * P, 0.0);
  for (int r = 0; r < P; ++r) {
    double diag = 0.0;
    for (int c = 0; c < P; ++c) {
      if (c == r) continue;
      D[r + (size_t)P * c] = bw[c] / (bw[r] * (ctrl[r] - ctrl[c]));
      diag = diag - D[r + (size_t)P * c];
    }
    D[r + (size_t)P * r] = diag;
  }
  for (int r = 0; r < P; ++r)
    for (int c = 0; c < P; ++c) {
      dM[c + (size_t)P * r] = D[r + (size_t)P * c];
      dgM[c + (size_t)P * r] = -D[c + (size_t)P * r] * qw[c] / qw[r];
    }
  basis_at(N, ctrl, bw, -1.0, bM);
  basis_at(N, ctrl, bw, 1.0, bM + P);
  return SELFGPU_OK;
}

namespace {
// local side -> its two CGNS corners (0-based), corners SW, SE, NE, NW
const int kSideCorners[4][2] = {{0, 1}, {1, 2}, {3, 2}, {0, 3}};
const int kCornerIJ[4][2] = {{0, 0}, {1, 0}, {1, 1}, {0, 1}};
}  // namespace

int mesh2d_structured(int nx, int ny, double x0, double x1, double y0, double y1, int perX, int perY, double amp,
                      int bcid, const int* rot, double* nodeCoords, int* gnid, int* sideInfo) {
  if (nx < 1 || ny < 1) return set_error(SELFGPU_ERR_ARG, "mesh2d_structured: nx, ny must be >= 1");
  // With one element across a periodic direction, both corners of the edges
  // along it are one node, and the flip of a rotated element's side could not
  // be read from the corner ids.
  if (rot && ((perX && nx == 1) || (perY && ny == 1)))
    for (int e = 0; e < nx * ny; ++e)
      if (((rot[e] % 4) + 4) % 4 != 0)
        return set_error(SELFGPU_ERR_ARG,
                         "mesh2d_structured: rotated elements need >= 2 elements across a periodic direction");
  const int nEl = nx * ny;
  const double hx = (x1 - x0) / nx, hy = (y1 - y0) / ny, h = std::min(hx, hy);
  const int rowLen = perX ? nx : nx + 1;
  auto node_id = [&](int ix, int iy) {
    if (perX) ix %= nx;
    if (perY) iy %= ny;
    return 1 + ix + rowLen * iy;
  };
  auto node_xy = [&](int ix, int iy, double* p) {
    p[0] = x0 + hx * (double)ix;
    p[1] = y0 + hy * (double)iy;
    if (amp != 0.0 && ix > 0 && ix < nx && iy > 0 && iy < ny) {
      double d = amp * h * std::sin(2.0 * kPi * (p[0] - x0) / (x1 - x0)) * std::sin(2.0 * kPi * (p[1] - y0) / (y1 - y0));
      p[0] += d;
      p[1] += d;
    }
  };
  for (int iy = 0; iy < ny; ++iy)
    for (int ix = 0; ix < nx; ++ix) {
      const int e = ix + nx * iy;
      const int r = rot ? ((rot[e] % 4) + 4) % 4 : 0;
      for (int c = 0; c < 4; ++c) {
        const int oc = (c + r) % 4;
        const int gx = ix + kCornerIJ[oc][0], gy = iy + kCornerIJ[oc][1];
        const int i = kCornerIJ[c][0], j = kCornerIJ[c][1];
        node_xy(gx, gy, nodeCoords + 2 * (i + 2 * (j + 2 * (size_t)e)));
        gnid[i + 2 * (j + 2 * (size_t)e)] = node_id(gx, gy);
      }
    }
  auto corner_id = [&](int e, int c) { return gnid[kCornerIJ[c][0] + 2 * (kCornerIJ[c][1] + 2 * (size_t)e)]; };
  // Sides are matched by the grid edge they lie on (orientation and lower-left
  // grid node, wrapped in the periodic directions) and ordered by their corner
  // ids.  The corner ids alone do not tell edges apart when a periodic
  // direction is one or two elements wide (the two edges of such a row share
  // both corner nodes).
  auto edge_code = [&](int e, int s) {
    const int ix = e % nx, iy = e / nx;
    const int r = rot ? ((rot[e] % 4) + 4) % 4 : 0;
    const int ca = (kSideCorners[s][0] + r) % 4, cb = (kSideCorners[s][1] + r) % 4;
    const int xa = ix + kCornerIJ[ca][0], ya = iy + kCornerIJ[ca][1];
    const int xb = ix + kCornerIJ[cb][0], yb = iy + kCornerIJ[cb][1];
    const int vertical = (xa == xb);
    int gx = std::min(xa, xb), gy = std::min(ya, yb);
    if (perX) gx %= nx;
    if (perY) gy %= ny;
    return 2 * (gx + (nx + 1) * gy) + vertical;
  };
  std::map<std::tuple<int, int, int>, std::vector<std::pair<int, int>>> faces;
  for (int e = 0; e < nEl; ++e)
    for (int s = 0; s < 4; ++s) {
      int a = corner_id(e, kSideCorners[s][0]), b = corner_id(e, kSideCorners[s][1]);
      faces[{std::min(a, b), std::max(a, b), edge_code(e, s)}].push_back({e, s});
    }
  int gid = 0;
  for (auto& kv : faces) {
    ++gid;
    const auto& v = kv.second;
    if (v.size() == 2) {
      for (int k = 0; k < 2; ++k) {
        int* si = sideInfo + 5 * (v[k].second + 4 * (size_t)v[k].first);
        const int e2 = v[1 - k].first, s2 = v[1 - k].second;
        // flip: 0 when the two sides list their shared corners in the same order
        const int a1 = corner_id(v[k].first, kSideCorners[v[k].second][0]);
        const int b1 = corner_id(v[k].first, kSideCorners[v[k].second][1]);
        const int a2 = corner_id(e2, kSideCorners[s2][0]);
        const int b2 = corner_id(e2, kSideCorners[s2][1]);
        const int flip = (std::abs(a1 - a2) + std::abs(b1 - b2) == 0) ? 0 : 1;
        si[0] = 1;
        si[1] = k == 0 ? gid : -gid;
        si[2] = e2 + 1;
        si[3] = 10 * (s2 + 1) + flip;
        si[4] = 0;
      }
    } else if (v.size() == 1) {
      int* si = sideInfo + 5 * (v[0].second + 4 * (size_t)v[0].first);
      si[0] = 1;
      si[1] = gid;
      si[2] = 0;
      si[3] = 0;
      si[4] = bcid;
    } else {
      return set_error(SELFGPU_ERR_MESH, "mesh2d_structured: a side is shared by more than two elements");
    }
  }
  return SELFGPU_OK;
}

int validate_side_info(const int* sideInfo, int nEl, int nNeighbours) {
  for (int e = 0; e < nEl; ++e)
    for (int s = 0; s < 4; ++s) {
      const int* si = sideInfo + 5 * (s + 4 * (size_t)e);
      const int e2 = si[2], s2 = si[3] / 10, flip = si[3] % 10, bcid = si[4];
      if (bcid == 0) {
        if (e2 < 1 || e2 > nNeighbours || s2 < 1 || s2 > 4 || (flip != 0 && flip != 1))
          return set_error(SELFGPU_ERR_MESH, "sideInfo: element " + std::to_string(e + 1) + " side " +
                                                 std::to_string(s + 1) + " has an invalid neighbour record");
      } else if (e2 < 0 || e2 > nNeighbours) {
        return set_error(SELFGPU_ERR_MESH, "sideInfo: element " + std::to_string(e + 1) + " side " +
                                               std::to_string(s + 1) + " has an out-of-range neighbour id");
      }
    }
  return SELFGPU_OK;
}

void modal_matrix(int N, const double* x, const double* w, double* T) {
  const int P = N + 1;
  for (int i = 0; i < P; ++i)
    for (int k = 0; k < P; ++k) {
      double l, dl;
      legendre(k, x[i], l, dl);
      T[k + P * i] = (std::sqrt((2.0 * k + 1.0) / 2.0) * l) * w[i];
    }
}

}  // namespace selfgpu

// ------------------------------------------------------------------ C ABI
extern "C" {

const char* selfgpu_last_error(void) { return selfgpu::last_error(); }

int selfgpu_legendre_quadrature(int N, int type, double* nodes, double* weights) {
  if (N < 0 || N > SELFGPU_MAX_N || !nodes || !weights)
    return selfgpu::set_error(SELFGPU_ERR_ARG, "selfgpu_legendre_quadrature: bad arguments");
  selfgpu::legendre_quadrature(N, type, nodes, weights);
  return SELFGPU_OK;
}

int selfgpu_lagrange_init(int N, int controlNodeType, int M, int targetNodeType, double* controlPoints,
                          double* targetPoints, double* bWeights, double* qWeights, double* iMatrix,
                          double* dMatrix, double* dgMatrix, double* bMatrix) {
  return selfgpu::lagrange_init(N, controlNodeType, M, targetNodeType, controlPoints, targetPoints, bWeights,
                                qWeights, iMatrix, dMatrix, dgMatrix, bMatrix);
}

int selfgpu_mesh2d_structured(int nx, int ny, double x0, double x1, double y0, double y1, int periodicX,
                              int periodicY, double perturbation, int bcid, const int* rotation,
                              double* nodeCoords, int* globalNodeIDs, int* sideInfo) {
  if (!nodeCoords || !globalNodeIDs || !sideInfo)
    return selfgpu::set_error(SELFGPU_ERR_ARG, "selfgpu_mesh2d_structured: null output");
  return selfgpu::mesh2d_structured(nx, ny, x0, x1, y0, y1, periodicX, periodicY, perturbation, bcid, rotation,
                                    nodeCoords, globalNodeIDs, sideInfo);
}

int selfgpu_modal_matrix(int N, const double* controlPoints, const double* qWeights, double* T) {
  if (N < 0 || N > SELFGPU_MAX_N || !controlPoints || !qWeights || !T)
    return selfgpu::set_error(SELFGPU_ERR_ARG, "selfgpu_modal_matrix: bad arguments");
  selfgpu::modal_matrix(N, controlPoints, qWeights, T);
  return SELFGPU_OK;
}

int selfgpu_validate_side_info(const int* sideInfo, int nEl) {
  if (!sideInfo || nEl < 1) return selfgpu::set_error(SELFGPU_ERR_ARG, "selfgpu_validate_side_info: bad arguments");
  return selfgpu::validate_side_info(sideInfo, nEl, nEl);
}

}  // extern "C"
