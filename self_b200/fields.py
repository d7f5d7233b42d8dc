"""SELF's field containers on the device: Scalar2D, Vector2D, MappedScalar2D,
MappedVector2D (src/SELF_Data.f90:86-178, src/SELF_MappedData.f90:37-103).

Each object holds the reference's arrays as device tensors in its Fortran
layouts (a Fortran array of shape (a, b, ..., nEl) is a contiguous tensor of
the reversed shape):

  Scalar2D   interior (P,P,nVar,nEl); boundary, extBoundary, avgBoundary
             (P,nVar,4,nEl)
  Vector2D   interior (2,P,P,nVar,nEl); boundary, extBoundary, avgBoundary
             (2,P,nVar,4,nEl); boundaryNormal (P,nVar,4,nEl)

and its type-bound procedures run the library's drop-in wrappers (the same
kernels SELF's `IF (gpuAccel)` branches reach), so code written against
SELF's Fortran field API -- f % BoundaryInterp(), f % SideExchange(mesh),
f % GradientBR(geometry, df), v % ContravariantProjection(geometry),
v % Divergence(geometry, dv) -- reads the same here.  Single-rank
exchanges only (rankId 0, offset 0); multi-rank runs use self_b200.decomp.
"""
import ctypes

import torch

from ._lib import check, lib, pp

_F64 = dict(device="cuda", dtype=torch.float64)


def _pp(t):
    return pp(t.data_ptr())


class Scalar2D:
    """src/SELF_Data.f90:86-104 (Init_Scalar2D :556-586)."""

    def __init__(self, interp, nVar, nElem):
        self.interp, self.nVar, self.nElem = interp, nVar, nElem
        self.N = interp.N
        P = self.N + 1
        self.interior = torch.zeros((nElem, nVar, P, P), **_F64)
        self.boundary = torch.zeros((nElem, 4, nVar, P), **_F64)
        self.extBoundary = torch.zeros((nElem, 4, nVar, P), **_F64)
        self.avgBoundary = torch.zeros((nElem, 4, nVar, P), **_F64)

    def BoundaryInterp(self):
        """BoundaryInterp_Scalar2D (src/SELF_Data.f90:630-647)."""
        lib().ScalarBoundaryInterp_2D_gpu_wrapper(_pp(self.interp.device("bMatrix")), _pp(self.interior),
                                                  _pp(self.boundary), self.N, self.nVar, self.nElem)

    def GridInterp(self, out):
        """GridInterp_Scalar2D (src/SELF_Data.f90:649-667): interior onto out's
        grid with interp % iMatrix (interp built with M = out's degree)."""
        lib().ScalarGridInterp_2D_gpu_wrapper(_pp(self.interp.device("iMatrix")), _pp(self.interior),
                                              _pp(out.interior), self.N, self.interp.M, self.nVar, self.nElem)


class Vector2D:
    """src/SELF_Data.f90:144-178 (Init_Vector2D :932-962)."""

    def __init__(self, interp, nVar, nElem):
        self.interp, self.nVar, self.nElem = interp, nVar, nElem
        self.N = interp.N
        P = self.N + 1
        self.interior = torch.zeros((nElem, nVar, P, P, 2), **_F64)
        self.boundary = torch.zeros((nElem, 4, nVar, P, 2), **_F64)
        self.extBoundary = torch.zeros((nElem, 4, nVar, P, 2), **_F64)
        self.avgBoundary = torch.zeros((nElem, 4, nVar, P, 2), **_F64)
        self.boundaryNormal = torch.zeros((nElem, 4, nVar, P), **_F64)

    def BoundaryInterp(self):
        """BoundaryInterp_Vector2D (src/SELF_Data.f90:1015-1032)."""
        lib().VectorBoundaryInterp_2D_gpu_wrapper(_pp(self.interp.device("bMatrix")), _pp(self.interior),
                                                  _pp(self.boundary), self.N, self.nVar, self.nElem)

    def GridInterp(self, out):
        """GridInterp_Vector2D (src/SELF_Data.f90:1034-1052)."""
        lib().VectorGridInterp_2D_gpu_wrapper(_pp(self.interp.device("iMatrix")), _pp(self.interior),
                                              _pp(out.interior), self.N, self.interp.M, self.nVar, self.nElem)


def _elem_to_rank(mesh):
    if not hasattr(mesh, "_elemToRank"):
        mesh._elemToRank = torch.zeros(mesh.nElem, device="cuda", dtype=torch.int32)
    return mesh._elemToRank


class MappedScalar2D(Scalar2D):
    """src/SELF_MappedData.f90:37-61."""

    def SideExchange(self, mesh):
        """SideExchange_MappedScalar2D (src/SELF_MappedData.f90:834-917): extBoundary
        of interior sides from the neighbours' boundary (flip applied); physical
        sides untouched."""
        lib().SideExchange_MappedScalar2D_gpu_wrapper(_pp(self.extBoundary), _pp(self.boundary),
                                                      pp(mesh.sideInfo_d.data_ptr()),
                                                      pp(_elem_to_rank(mesh).data_ptr()), 0, 0, self.N, self.nVar,
                                                      self.nElem)

    def BassiRebaySides(self):
        """BassiRebaySides_MappedScalar2D (src/SELF_MappedData.f90:919-953)."""
        lib().BassiRebaySides_MappedScalar2D_gpu_wrapper(_pp(self.avgBoundary), _pp(self.boundary),
                                                         _pp(self.extBoundary), self.N, self.nVar, self.nElem)

    def GradientSF(self, geometry, gradF):
        """GradientSF_MappedScalar2D (src/SELF_MappedData.f90:1080-1149) into gradF % interior."""
        lib().GradientSF_MappedScalar2D_gpu_wrapper(_pp(self.interior), _pp(geometry.dsdx), _pp(geometry.J),
                                                    _pp(gradF.interior), _pp(self.interp.device("dMatrix")),
                                                    self.N, self.nVar, self.nElem)

    def GradientBR(self, geometry, gradF):
        """GradientBR_MappedScalar2D (src/SELF_MappedData.f90:955-1078): the weak
        gradient with the avgBoundary lift (call BoundaryInterp, SideExchange
        and BassiRebaySides first, as the reference does)."""
        L = self.interp
        lib().GradientBR_MappedScalar2D_gpu_wrapper(_pp(self.interior), _pp(self.avgBoundary), _pp(geometry.dsdx),
                                                    _pp(geometry.J), _pp(geometry.nHat), _pp(geometry.nScale),
                                                    _pp(gradF.interior), _pp(L.device("dgMatrix")),
                                                    _pp(L.device("bMatrix")), _pp(L.device("qWeights")), self.N,
                                                    self.nVar, self.nElem)

    def JacobianWeight(self, geometry):
        """JacobianWeight_MappedScalar2D (src/SELF_MappedData.f90:1235-1268): interior / J."""
        lib().JacobianWeight_MappedScalar2D_gpu_wrapper(_pp(self.interior), _pp(geometry.J), self.N, self.nVar,
                                                        self.nElem)

    def Integral(self, geometry, iVar=4):
        """Integral_MappedScalar2D (src/SELF_MappedData.f90:1270-1311): sum of
        f J w_i w_j over the mesh, reduced on the device.  The reference
        integrates variable 4 (hard-coded); iVar (1-based) defaults to it."""
        if not 1 <= iVar <= self.nVar:
            raise ValueError(f"iVar must be in 1..{self.nVar}")
        out = ctypes.c_double()
        qw = self.interp.qWeights
        check(lib().selfgpu_integral_mapped_scalar2d(ctypes.c_void_p(self.interior.data_ptr()), iVar, self.nVar,
                                                     ctypes.c_void_p(geometry.J.data_ptr()),
                                                     qw.ctypes.data_as(ctypes.c_void_p), self.N, self.nElem,
                                                     ctypes.byref(out), None))
        return out.value


class MappedVector2D(Vector2D):
    """src/SELF_MappedData.f90:79-103."""

    def SideExchange(self, mesh):
        """SideExchange_MappedVector2D (src/SELF_MappedData.f90:1870-1958)."""
        lib().SideExchange_MappedVector2D_gpu_wrapper(_pp(self.extBoundary), _pp(self.boundary),
                                                      pp(mesh.sideInfo_d.data_ptr()),
                                                      pp(_elem_to_rank(mesh).data_ptr()), 0, 0, self.N, self.nVar,
                                                      self.nElem)

    def ContravariantProjection(self, geometry):
        """ContravariantProjection_MappedVector2D (src/SELF_MappedData.f90:2220-2269)."""
        lib().ContravariantProjection_MappedVector2D_gpu_wrapper(_pp(self.interior), _pp(geometry.dsdx), self.N,
                                                                 self.nVar, self.nElem)

    def JacobianWeight(self, geometry):
        """JacobianWeight_MappedVector2D (src/SELF_MappedData.f90:2271-2306)."""
        lib().JacobianWeight_MappedVector2D_gpu_wrapper(_pp(self.interior), _pp(geometry.J), self.N, self.nVar,
                                                        self.nElem)

    def Divergence(self, geometry, divVector):
        """Divergence_MappedVector2D, weak DG form (src/SELF_MappedData.f90:1996-2044):
        VectorDGDivergence_2D of the (already projected) interior with
        boundaryNormal, then divVector % JacobianWeight."""
        L = self.interp
        lib().VectorDGDivergence_2D_gpu_wrapper(_pp(L.device("dgMatrix")), _pp(L.device("bMatrix")),
                                                _pp(L.device("qWeights")), _pp(self.interior),
                                                _pp(self.boundaryNormal), _pp(divVector.interior), self.N, self.nVar,
                                                self.nElem)
        divVector.JacobianWeight(geometry)


__all__ = ["Scalar2D", "Vector2D", "MappedScalar2D", "MappedVector2D"]
