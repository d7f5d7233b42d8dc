"""ctypes front end of the FP64 CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module.  It wraps ``self_oracle.cpp``, the restatement of the reference's
CPU branches; array shapes are returned in Fortran order (``order='F'``) so
``a[i, j, v, e]`` reads like the reference's ``interior(i,j,v,e)`` with 0-based
v and e.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

GAUSS, GAUSS_LOBATTO, CHEBYSHEV_GAUSS, CHEBYSHEV_GAUSS_LOBATTO, UNIFORM = 1, 2, 3, 4, 5
BC_PRESCRIBED, BC_RADIATION, BC_NONORMALFLOW = 100, 101, 102
LSW, SW, CIG = 1, 2, 3

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_libs = {}


def lib(fast: bool = False):
    name = "liboracle_fast.so" if fast else "liboracle.so"
    if name not in _libs:
        path = os.path.join(HERE, "_build", name)
        if not os.path.exists(path):
            from oracle import build as _build
            _build.build()
        L = ctypes.CDLL(path)
        L.orc_model_create.restype = ctypes.c_void_p
        L.orc_model_entropy.restype = ctypes.c_double
        L.orc_model_arcmin.restype = ctypes.c_double
        L.orc_geometry.restype = ctypes.c_double
        L.orc_model_field_size.restype = ctypes.c_longlong
        for fn in ("orc_model_free", "orc_model_tendency", "orc_model_rk3", "orc_model_set",
                   "orc_model_get", "orc_model_set_params", "orc_model_entropy",
                   "orc_model_arcmin", "orc_model_field_size", "orc_model_set_closure"):
            getattr(L, fn).argtypes = None
        _libs[name] = L
    return _libs[name]


def _p(a):
    if a is None:
        return None
    if a.dtype == np.int32:
        return a.ctypes.data_as(_I)
    return a.ctypes.data_as(_D)


def _z(*shape):
    return np.zeros(shape, dtype=np.float64, order="F")


def quadrature(N, qtype=GAUSS):
    x, w = _z(N + 1), _z(N + 1)
    lib().orc_legendre_quadrature(N, qtype, _p(x), _p(w))
    return x, w


class Lagrange:
    """Lagrange%Init outputs (src/SELF_Lagrange.f90:521-615)."""

    def __init__(self, N, ctrl=GAUSS, M=None, tgt=UNIFORM):
        M = N if M is None else M
        self.N, self.M = N, M
        P, Q = N + 1, M + 1
        self.controlPoints, self.targetPoints = _z(P), _z(Q)
        self.bWeights, self.qWeights = _z(P), _z(P)
        self.iMatrix, self.dMatrix, self.dgMatrix, self.bMatrix = _z(P, Q), _z(P, P), _z(P, P), _z(P, 2)
        lib().orc_lagrange(N, ctrl, M, tgt, _p(self.controlPoints), _p(self.targetPoints),
                           _p(self.bWeights), _p(self.qWeights), _p(self.iMatrix), _p(self.dMatrix),
                           _p(self.dgMatrix), _p(self.bMatrix))


# ---- single operators on raw Fortran-layout arrays
def scalar_boundary_interp(L, f):
    P, nVar, nEl = f.shape[0], f.shape[2], f.shape[3]
    fb = _z(P, nVar, 4, nEl)
    lib().orc_scalar_boundary_interp_2d(_p(L.bMatrix), _p(f), _p(fb), P - 1, nVar, nEl)
    return fb


def vector_boundary_interp(L, f):
    P, nVar, nEl = f.shape[1], f.shape[3], f.shape[4]
    fb = _z(2, P, nVar, 4, nEl)
    lib().orc_vector_boundary_interp_2d(_p(L.bMatrix), _p(f), _p(fb), P - 1, nVar, nEl)
    return fb


def tensor_boundary_interp(L, f):
    P, nVar, nEl = f.shape[2], f.shape[4], f.shape[5]
    fb = _z(2, 2, P, nVar, 4, nEl)
    lib().orc_tensor_boundary_interp_2d(_p(L.bMatrix), _p(f), _p(fb), P - 1, nVar, nEl)
    return fb


def scalar_grid_interp(L, f):
    P, nVar, nEl = f.shape[0], f.shape[2], f.shape[3]
    Q = L.M + 1
    fo = _z(Q, Q, nVar, nEl)
    lib().orc_scalar_grid_interp_2d(_p(L.iMatrix), _p(f), _p(fo), P - 1, L.M, nVar, nEl)
    return fo


def vector_grid_interp(L, f):
    P, nVar, nEl = f.shape[1], f.shape[3], f.shape[4]
    Q = L.M + 1
    fo = _z(2, Q, Q, nVar, nEl)
    lib().orc_vector_grid_interp_2d(_p(L.iMatrix), _p(f), _p(fo), P - 1, L.M, nVar, nEl)
    return fo


def vector_gradient(L, f):
    P, nVar, nEl = f.shape[1], f.shape[3], f.shape[4]
    g = _z(2, 2, P, P, nVar, nEl)
    lib().orc_vector_gradient_2d(_p(L.dMatrix), _p(f), _p(g), P - 1, nVar, nEl)
    return g


def vector_dg_divergence(L, f, bf):
    P, nVar, nEl = f.shape[1], f.shape[3], f.shape[4]
    df = _z(P, P, nVar, nEl)
    lib().orc_vector_dg_divergence_2d(_p(L.dgMatrix), _p(L.bMatrix), _p(L.qWeights), _p(f), _p(bf),
                                      _p(df), P - 1, nVar, nEl)
    return df


def jacobian_weight(f, J):
    f = np.array(f, order="F", copy=True)
    P, nVar, nEl = f.shape[0], f.shape[2], f.shape[3]
    lib().orc_jacobian_weight_2d(_p(f), _p(J), P - 1, nVar, nEl)
    return f


def contravariant_projection(f, dsdx):
    f = np.array(f, order="F", copy=True)
    P, nVar, nEl = f.shape[1], f.shape[3], f.shape[4]
    lib().orc_contravariant_projection_2d(_p(f), _p(dsdx), P - 1, nVar, nEl)
    return f


def side_exchange_scalar(bnd, sideInfo, ext=None):
    ext = _z(*bnd.shape) if ext is None else np.array(ext, order="F", copy=True)
    P, nVar, nEl = bnd.shape[0], bnd.shape[1], bnd.shape[3]
    lib().orc_side_exchange_scalar_2d(_p(ext), _p(bnd), _p(sideInfo), P - 1, nVar, nEl)
    return ext


def side_exchange_vector(bnd, sideInfo, ext=None):
    ext = _z(*bnd.shape) if ext is None else np.array(ext, order="F", copy=True)
    P, nVar, nEl = bnd.shape[1], bnd.shape[2], bnd.shape[4]
    lib().orc_side_exchange_vector_2d(_p(ext), _p(bnd), _p(sideInfo), P - 1, nVar, nEl)
    return ext


def bassi_rebay_sides(bnd, ext):
    avg = _z(*bnd.shape)
    P, nVar, nEl = bnd.shape[0], bnd.shape[1], bnd.shape[3]
    lib().orc_bassi_rebay_sides_2d(_p(avg), _p(bnd), _p(ext), P - 1, nVar, nEl)
    return avg


def gradient_sf(L, f, dsdx, J):
    P, nVar, nEl = f.shape[0], f.shape[2], f.shape[3]
    g = _z(2, P, P, nVar, nEl)
    lib().orc_gradient_sf_2d(_p(f), _p(dsdx), _p(J), _p(g), _p(L.dMatrix), P - 1, nVar, nEl)
    return g


def gradient_br(L, f, avgB, dsdx, J, nHat, nScale):
    P, nVar, nEl = f.shape[0], f.shape[2], f.shape[3]
    g = _z(2, P, P, nVar, nEl)
    lib().orc_gradient_br_2d(_p(f), _p(avgB), _p(dsdx), _p(J), _p(nHat), _p(nScale), _p(g),
                             _p(L.dgMatrix), _p(L.bMatrix), _p(L.qWeights), P - 1, nVar, nEl)
    return g


def determinant(t):
    P, nVar, nEl = t.shape[2], t.shape[4], t.shape[5]
    d = _z(P, P, nVar, nEl)
    lib().orc_determinant_2d(_p(t), _p(d), P - 1, nVar, nEl)
    return d


# ---- mesh and geometry
class Mesh:
    """Structured quadrilateral mesh (nGeo = 1) with SELF sideInfo conventions."""

    def __init__(self, nx, ny, x0=0.0, x1=1.0, y0=0.0, y1=1.0, periodic=(False, False), amp=0.0,
                 bcid=BC_NONORMALFLOW, rot=None):
        self.nx, self.ny, self.nEl = nx, ny, nx * ny
        self.nodeCoords = _z(2, 2, 2, self.nEl)
        self.globalNodeIDs = np.zeros((2, 2, self.nEl), dtype=np.int32, order="F")
        self.sideInfo = np.zeros((5, 4, self.nEl), dtype=np.int32, order="F")
        r = None if rot is None else np.ascontiguousarray(rot, dtype=np.int32)
        lib().orc_mesh_structured(nx, ny, ctypes.c_double(x0), ctypes.c_double(x1), ctypes.c_double(y0),
                                  ctypes.c_double(y1), int(periodic[0]), int(periodic[1]),
                                  ctypes.c_double(amp), bcid, _p(r), _p(self.nodeCoords),
                                  _p(self.globalNodeIDs), _p(self.sideInfo))


class Geometry:
    """SEMQuad%GenerateFromMesh outputs (src/SELF_Geometry.f90:393-552)."""

    def __init__(self, N, mesh, quad=GAUSS):
        P, nEl = N + 1, mesh.nEl
        self.x, self.xB = _z(2, P, P, 1, nEl), _z(2, P, 1, 4, nEl)
        self.dxds, self.dxdsB = _z(2, 2, P, P, 1, nEl), _z(2, 2, P, 1, 4, nEl)
        self.dsdx, self.dsdxB = _z(2, 2, P, P, 1, nEl), _z(2, 2, P, 1, 4, nEl)
        self.J, self.JB = _z(P, P, 1, nEl), _z(P, 1, 4, nEl)
        self.nHat, self.nScale = _z(2, P, 1, 4, nEl), _z(P, 1, 4, nEl)
        self.arcmin = lib().orc_geometry(N, quad, nEl, _p(mesh.nodeCoords), _p(self.x), _p(self.xB),
                                         _p(self.dxds), _p(self.dxdsB), _p(self.dsdx), _p(self.dsdxB),
                                         _p(self.J), _p(self.JB), _p(self.nHat), _p(self.nScale))


class Model:
    """Model2D + physics (LSW / SW / CIG) as restated in self_oracle.cpp."""

    NVAR = {LSW: 3, SW: 3, CIG: 4}

    def __init__(self, kind, N, mesh, quad=GAUSS, g=1.0, fCori=0.0, Cp=1.4, Cv=1.0, R=1.0, fast=False):
        self.kind, self.N, self.nEl, self.nVar = kind, N, mesh.nEl, self.NVAR[kind]
        self.L = lib(fast)
        self.h = ctypes.c_void_p(self.L.orc_model_create(kind, N, quad, mesh.nEl, _p(mesh.sideInfo),
                                                         _p(mesh.nodeCoords)))
        self.L.orc_model_set_params(self.h, ctypes.c_double(g), ctypes.c_double(fCori), ctypes.c_double(Cp),
                                    ctypes.c_double(Cv), ctypes.c_double(R))

    def __del__(self):
        try:
            self.L.orc_model_free(self.h)
        except Exception:
            pass

    def set(self, name, data=None):
        d = None if data is None else np.asfortranarray(data, dtype=np.float64)
        rc = self.L.orc_model_set(self.h, name.encode(), _p(d))
        if rc != 0:
            raise KeyError(name)

    def get(self, name, shape=None):
        n = self.L.orc_model_field_size(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n, dtype=np.float64)
        self.L.orc_model_get(self.h, name.encode(), _p(out))
        return out if shape is None else out.reshape(shape, order="F")

    def interior_shape(self, nv=None):
        P = self.N + 1
        return (P, P, self.nVar if nv is None else nv, self.nEl)

    def tendency(self):
        self.L.orc_model_tendency(self.h)
        return self.get("dSdt", self.interior_shape())

    def rk3(self, n_steps, dt):
        self.L.orc_model_rk3(self.h, int(n_steps), ctypes.c_double(dt))

    def entropy(self):
        return self.L.orc_model_entropy(self.h)

    def arcmin(self):
        return self.L.orc_model_arcmin(self.h)

    def set_closure(self, mode, c=1.0, s0=None, kappa=1.0):
        """Artificial-viscosity closure (CIG): 0 off, 1 modal-decay indicator,
        2 element viscosity given through set("avNu", ...)."""
        if s0 is None:
            s0 = default_s0(self.N)
        rc = self.L.orc_model_set_closure(self.h, int(mode), ctypes.c_double(c), ctypes.c_double(s0),
                                          ctypes.c_double(kappa))
        if rc != 0:
            raise ValueError("closure needs a CompressibleIdealGas2D model")


def default_s0(N):
    """Indicator threshold s0 = log10(1/N^4) (Persson & Peraire)."""
    return float(-4.0 * np.log10(N))


def modal_matrix(N, quad=GAUSS):
    T = _z(N + 1, N + 1)
    lib().orc_modal_matrix(N, quad, _p(T))
    return T


def closure_features(q, N, s0=None, kappa=1.0, quad=GAUSS):
    """Modal-decay activation of the density (nEl,) and the 36 closure
    features (36, nEl) of a (P,P,4,nEl) CompressibleIdealGas2D state."""
    q = np.asfortranarray(q, dtype=np.float64)
    nEl = q.shape[3]
    T = modal_matrix(N, quad)
    act, feat = np.zeros(nEl), _z(36, nEl)
    if s0 is None:
        s0 = default_s0(N)
    lib().orc_closure_features(_p(T), _p(q), int(N), int(nEl), ctypes.c_double(s0), ctypes.c_double(kappa),
                               _p(act), _p(feat))
    return act, feat


def bf16_round(x):
    """Round float32 values to bfloat16 (nearest, ties to even), returned as float32."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return (b.astype(np.uint32) << 16).view(np.float32).reshape(np.shape(x))


def mlp_forward(feat, W1, b1, W2, b2, w3, b3):
    """Closure MLP 36 -> 32 -> 32 -> 1 with bfloat16 weights and float32
    accumulation; output clamp(z, 0, 1).  feat is (36, n); returns (n,)."""
    f = np.asarray(feat, dtype=np.float32)
    h1 = np.maximum(bf16_round(W1) @ f + np.asarray(b1, np.float32)[:, None], 0)
    h2 = np.maximum(bf16_round(W2) @ h1 + np.asarray(b2, np.float32)[:, None], 0)
    z = bf16_round(np.asarray(w3, np.float32)) @ h2 + np.float32(b3)
    return np.clip(z, 0.0, 1.0)


def set_threads(n, fast=False):
    return lib(fast).orc_set_threads(int(n))
