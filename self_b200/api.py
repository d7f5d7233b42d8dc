"""Host-side mirror of SELF's 2-D API over libselfgpu's C ABI.

The classes keep the reference's names and call order -- ``Lagrange``,
``Mesh2D``, ``SEMQuad``, ``Model2D`` and the three 2-D models with
``SetSolution``, ``CalculateTendency``, ``ForwardStep`` -- so a script written
against SELF's Fortran API (src/SELF_Model2D.f90, src/models/*.f90) reads the
same here.  All compute runs in the CUDA library: set-up operators through the
drop-in wrappers (BoundaryInterp, GradientSF, diagnostics) and the time loop
through the fused engine.  PyTorch only holds device memory.

Device arrays use the reference's Fortran layouts; a Fortran array of shape
``(P, P, nVar, nEl)`` is held as a contiguous tensor of the reversed shape
``(nEl, nVar, P, P)`` (identical memory).  ``to_device``/``to_host`` convert.
"""
import ctypes

import numpy as np
import torch

from ._lib import check, lib, pp

GAUSS, GAUSS_LOBATTO, UNIFORM = 1, 2, 5
BC_PRESCRIBED, BC_RADIATION, BC_NONORMALFLOW = 100, 101, 102
MODEL_LSW, MODEL_SW, MODEL_CIG = 1, 2, 3
# arithmetic forms: FP64 = production FP64 (contraction, reciprocal products),
# FP32_BULK = FP32 fluxes/divergence, FP64_REF = FP64 with the reference's roundings
FP64, FP32_BULK, FP64_REF = 0, 1, 2


def to_device(a, dtype=torch.float64, device="cuda"):
    """Fortran-ordered numpy array -> contiguous device tensor of reversed shape."""
    a = np.asfortranarray(a)
    return torch.from_numpy(np.ascontiguousarray(a.T)).to(device=device, dtype=dtype)


def to_host(t):
    """Device tensor of reversed shape -> Fortran-ordered numpy array."""
    return t.detach().cpu().numpy().T


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


CLOSURE_OFF, CLOSURE_INDICATOR, CLOSURE_MLP = 0, 1, 2


def default_s0(N):
    """Modal-decay threshold s0 = log10(1 / N^4) (Persson & Peraire)."""
    return float(-4.0 * np.log10(N))


class Lagrange:
    """Lagrange%Init (src/SELF_Lagrange.f90:521-615), built on the host."""

    def __init__(self, N, controlNodeType=GAUSS, M=None, targetNodeType=UNIFORM):
        M = N if M is None else M
        self.N, self.M, self.controlNodeType, self.targetNodeType = N, M, controlNodeType, targetNodeType
        P, Q = N + 1, M + 1
        z = lambda *s: np.zeros(s, dtype=np.float64, order="F")  # noqa: E731
        self.controlPoints, self.targetPoints, self.bWeights, self.qWeights = z(P), z(Q), z(P), z(P)
        self.iMatrix, self.dMatrix, self.dgMatrix, self.bMatrix = z(P, Q), z(P, P), z(P, P), z(P, 2)
        args = [self.controlPoints, self.targetPoints, self.bWeights, self.qWeights, self.iMatrix, self.dMatrix,
                self.dgMatrix, self.bMatrix]
        check(lib().selfgpu_lagrange_init(N, controlNodeType, M, targetNodeType,
                                          *[a.ctypes.data_as(ctypes.c_void_p) for a in args]))
        self._dev = {}

    def device(self, name):
        """Device copy of one of the operator arrays (for the drop-in wrappers)."""
        if name not in self._dev:
            self._dev[name] = to_device(getattr(self, name))
        return self._dev[name]


class Mesh2D:
    """Mesh2D connectivity (src/SELF_Mesh.f90:228-254) from the structured generator."""

    def __init__(self, nx, ny, x0=0.0, x1=1.0, y0=0.0, y1=1.0, periodic=(False, False), perturbation=0.0,
                 bcid=BC_RADIATION, rotation=None):
        self.nx, self.ny, self.nElem, self.nGeo = nx, ny, nx * ny, 1
        nEl = self.nElem
        self.nodeCoords = np.zeros((2, 2, 2, nEl), dtype=np.float64, order="F")
        self.globalNodeIDs = np.zeros((2, 2, nEl), dtype=np.int32, order="F")
        self.sideInfo = np.zeros((5, 4, nEl), dtype=np.int32, order="F")
        rot = None if rotation is None else np.ascontiguousarray(rotation, dtype=np.int32)
        check(lib().selfgpu_mesh2d_structured(
            nx, ny, x0, x1, y0, y1, int(periodic[0]), int(periodic[1]), perturbation, bcid,
            None if rot is None else rot.ctypes.data_as(ctypes.c_void_p),
            self.nodeCoords.ctypes.data_as(ctypes.c_void_p), self.globalNodeIDs.ctypes.data_as(ctypes.c_void_p),
            self.sideInfo.ctypes.data_as(ctypes.c_void_p)))
        self._upload()

    @classmethod
    def from_arrays(cls, nodeCoords, sideInfo):
        m = cls.__new__(cls)
        m.nodeCoords = np.asfortranarray(nodeCoords, dtype=np.float64)
        m.sideInfo = np.asfortranarray(sideInfo, dtype=np.int32)
        m.nElem, m.nGeo = m.sideInfo.shape[2], 1
        m._upload()
        return m

    def _upload(self):
        # device copies are made on first use, so meshes can be built without a GPU
        self._dev = {}

    @property
    def sideInfo_d(self):
        if "sideInfo" not in self._dev:
            self._dev["sideInfo"] = to_device(self.sideInfo, dtype=torch.int32)
        return self._dev["sideInfo"]

    @property
    def nodeCoords_d(self):
        if "nodeCoords" not in self._dev:
            self._dev["nodeCoords"] = to_device(self.nodeCoords)
        return self._dev["nodeCoords"]

    def ResetBoundaryConditionType(self, bcid):
        """src/SELF_Mesh.f90:695-719: every physical side (no neighbour) gets bcid."""
        phys = self.sideInfo[2, :, :] == 0
        self.sideInfo[4, :, :][phys] = bcid
        self._upload()


class SEMQuad:
    """SEMQuad%GenerateFromMesh (src/SELF_Geometry.f90:393-552), computed on the device."""

    def __init__(self, interp, mesh):
        self.interp, self.nElem = interp, mesh.nElem
        N, P, nEl = interp.N, interp.N + 1, mesh.nElem
        m2m = Lagrange(mesh.nGeo, UNIFORM, N, interp.controlNodeType)
        dev = dict(device="cuda", dtype=torch.float64)
        self.x = torch.empty((nEl, 1, P, P, 2), **dev)
        self.dxds = torch.empty((nEl, 1, P, P, 2, 2), **dev)
        self.dsdx = torch.empty((nEl, 1, P, P, 2, 2), **dev)
        self.J = torch.empty((nEl, 1, P, P), **dev)
        self.dsdxBoundary = torch.empty((nEl, 4, 1, P, 2, 2), **dev)
        self.JBoundary = torch.empty((nEl, 4, 1, P), **dev)
        self.nHat = torch.empty((nEl, 4, 1, P, 2), **dev)
        self.nScale = torch.empty((nEl, 4, 1, P), **dev)
        self._keep = [np.asfortranarray(m2m.iMatrix), np.asfortranarray(interp.dMatrix),
                      np.asfortranarray(interp.bMatrix)]
        check(lib().selfgpu_semquad_generate(
            N, nEl, _ptr(mesh.nodeCoords_d), self._keep[0].ctypes.data_as(ctypes.c_void_p),
            self._keep[1].ctypes.data_as(ctypes.c_void_p), self._keep[2].ctypes.data_as(ctypes.c_void_p),
            _ptr(self.x), _ptr(self.dxds), _ptr(self.dsdx), _ptr(self.J), _ptr(self.dsdxBoundary),
            _ptr(self.JBoundary), _ptr(self.nHat), _ptr(self.nScale), None))

    def CovariantArcMin(self):
        """src/SELF_Geometry.f90:554-582."""
        N = self.interp.N
        d = self.dxds
        dx = torch.sqrt(d[..., 0, 0] ** 2 + d[..., 1, 0] ** 2)  # dxds(1,1), dxds(1,2)
        dy = torch.sqrt(d[..., 0, 1] ** 2 + d[..., 1, 1] ** 2)  # dxds(2,1), dxds(2,2)
        return float((2.0 * torch.minimum(dx, dy) / float(N * N)).min())


class Model2D:
    """Model2D on the fused engine (src/SELF_Model2D.f90)."""

    NVAR = {MODEL_LSW: 3, MODEL_SW: 3, MODEL_CIG: 4}

    def __init__(self, model_id, mesh, geometry, form=FP64, stream=None):
        self.model_id, self.mesh, self.geometry, self.form = model_id, mesh, geometry, form
        self.interp = geometry.interp
        self.N, self.nElem, self.nVar = self.interp.N, mesh.nElem, self.NVAR[model_id]
        P, nEl, nVar = self.N + 1, self.nElem, self.nVar
        dev = dict(device="cuda", dtype=torch.float64)
        self.solution = torch.zeros((nEl, nVar, P, P), **dev)
        self.workSol = torch.zeros((nEl, nVar, P, P), **dev)  # zeroed (the reference never uploads it)
        self.dSdt = torch.zeros((nEl, nVar, P, P), **dev)
        self.t, self.dt = 0.0, 0.0
        self.g, self.fCori, self.expansionFactor, self.R = 1.0, 0.0, 1.4, 1.0
        h = ctypes.c_void_p()
        check(lib().selfgpu_model2d_create(ctypes.byref(h), model_id, self.N, nEl, form,
                                           None if stream is None else ctypes.c_void_p(stream)))
        self._h = h
        L = self.interp
        self._mats = [np.asfortranarray(L.dgMatrix), np.asfortranarray(L.bMatrix), np.asfortranarray(L.qWeights)]
        check(lib().selfgpu_model2d_set_interp(h, *[a.ctypes.data_as(ctypes.c_void_p) for a in self._mats]))
        self.nHalo = int(getattr(mesh, "nHalo", 0))  # halo elements of a decomposed run (self_b200.decomp)
        if self.nHalo:
            check(lib().selfgpu_model2d_set_halo(h, self.nHalo))
        self._sideInfo_h = np.asfortranarray(mesh.sideInfo)
        check(lib().selfgpu_model2d_set_geometry(h, _ptr(geometry.dsdx), _ptr(geometry.J), _ptr(geometry.nHat),
                                                 _ptr(geometry.nScale), _ptr(mesh.sideInfo_d),
                                                 self._sideInfo_h.ctypes.data_as(ctypes.c_void_p)))
        check(lib().selfgpu_model2d_set_state(h, _ptr(self.solution), _ptr(self.workSol)))
        self._fields = {}
        self._push_params()

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().selfgpu_model2d_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ---- parameters and fields
    @property
    def g(self):
        """Acceleration of gravity (the reference's `model % g`); assigning it
        updates the engine's parameters."""
        return self._g

    @g.setter
    def g(self, value):
        self._g = float(value)
        if getattr(self, "_h", None) is not None:
            self._push_params()

    def _push_params(self):
        check(lib().selfgpu_model2d_set_params(self._h, self.g, self.fCori, self.expansionFactor, self.R))

    def _set_field(self, name, tensor):
        # Set-up fields are produced by drop-in wrappers on the legacy default
        # stream; finish them before a handle on another stream can read them.
        torch.cuda.synchronize()
        self._fields[name] = tensor
        check(lib().selfgpu_model2d_set_field(self._h, name.encode(), None if tensor is None else _ptr(tensor)))

    def _bnd_interp(self, interior, nVar):
        P, nEl = self.N + 1, self.nElem
        out = torch.zeros((nEl, 4, nVar, P), device="cuda", dtype=torch.float64)
        lib().ScalarBoundaryInterp_2D_gpu_wrapper(pp(self.interp.device("bMatrix").data_ptr()),
                                                  pp(interior.data_ptr()), pp(out.data_ptr()), self.N, nVar, nEl)
        return out

    def _gradient_sf(self, interior, nVar):
        P, nEl = self.N + 1, self.nElem
        out = torch.zeros((nEl, nVar, P, P, 2), device="cuda", dtype=torch.float64)
        lib().GradientSF_MappedScalar2D_gpu_wrapper(pp(interior.data_ptr()), pp(self.geometry.dsdx.data_ptr()),
                                                    pp(self.geometry.J.data_ptr()), pp(out.data_ptr()),
                                                    pp(self.interp.device("dMatrix").data_ptr()), self.N, nVar,
                                                    self.nElem)
        return out

    # ---- reference API
    def SetSolution(self, values):
        """Set the solution interior (Fortran-ordered array or reversed-shape tensor)."""
        t = values if isinstance(values, torch.Tensor) else to_device(values)
        self.solution.copy_(t.reshape(self.solution.shape))
        check(lib().selfgpu_model2d_invalidate(self._h))

    def CalculateTendency(self):
        check(lib().selfgpu_model2d_tendency(self._h, _ptr(self.dSdt)))
        return self.dSdt

    def ForwardStep(self, nSteps, dt=None):
        """nSteps RK3 steps of size dt (LowStorageRK3_timeIntegrator, stepped by count)."""
        if dt is not None:
            self.dt = dt
        check(lib().selfgpu_model2d_rk3(self._h, float(self.dt), int(nSteps)))
        self.t += nSteps * self.dt

    def Sync(self):
        check(lib().selfgpu_model2d_sync(self._h))

    def Write(self, fileName=None):
        """Write_Model2D (src/SELF_Model2D.f90:861-1058) to a checkpoint file; returns its name."""
        from .checkpoint import write_model
        return write_model(self, fileName)

    def Read(self, fileName, firstElem=0):
        """Read_Model2D (src/SELF_Model2D.f90:1060-1099): pickup of the solution."""
        from .checkpoint import read_model
        return read_model(self, fileName, firstElem)

    def CheckFinite(self):
        check(lib().selfgpu_model2d_check_finite(self._h))

    def CalculateEntropy(self):
        """CalculateEntropy of the model (src/models/SELF_*.f90), reduced on the
        device; kept in self.entropy as the reference keeps it."""
        e = ctypes.c_double()
        check(lib().selfgpu_model2d_entropy(self._h, ctypes.byref(e)))
        self.entropy = e.value
        return self.entropy

    def LaunchCount(self):
        return lib().selfgpu_model2d_launch_count(self._h)

    def _wJ(self):
        w = torch.as_tensor(self.interp.qWeights, device="cuda")
        return self.geometry.J[:, 0] * w[None, None, :] * w[None, :, None]


class LinearShallowWater(Model2D):
    """src/models/SELF_LinearShallowWater.f90."""

    def __init__(self, mesh, geometry, form=FP64, stream=None):
        super().__init__(MODEL_LSW, mesh, geometry, form, stream)
        self.SetBathymetry(1.0)

    def SetBathymetry(self, H):
        P, nEl = self.N + 1, self.nElem
        Hi = torch.full((nEl, 1, P, P), float(H), device="cuda", dtype=torch.float64) if np.isscalar(H) else \
            (H if isinstance(H, torch.Tensor) else to_device(H)).reshape(nEl, 1, P, P).contiguous()
        self._set_field("H", Hi)
        self._set_field("H.boundary", self._bnd_interp(Hi, 1))

    def SetCoriolis(self, f):
        P, nEl = self.N + 1, self.nElem
        fi = (f if isinstance(f, torch.Tensor) else to_device(f)).reshape(nEl, 1, P, P).contiguous()
        self._set_field("fCori", fi)



class ShallowWater(Model2D):
    """src/models/SELF_ShallowWater.f90 (device path is new; the reference runs it on the CPU)."""

    def __init__(self, mesh, geometry, form=FP64, stream=None):
        super().__init__(MODEL_SW, mesh, geometry, form, stream)
        P, nEl = self.N + 1, self.nElem
        self.SetTopography(torch.zeros((nEl, 1, P, P), device="cuda", dtype=torch.float64))

    def SetTopography(self, h):
        P, nEl = self.N + 1, self.nElem
        hi = (h if isinstance(h, torch.Tensor) else to_device(h)).reshape(nEl, 1, P, P).contiguous()
        self.topography = hi
        self._set_field("topography", hi)
        self._set_field("topography.boundary", self._bnd_interp(hi, 1))
        self._set_field("gradTopography", self._gradient_sf(hi, 1))



class CompressibleIdealGas2D(Model2D):
    """src/models/SELF_CompressibleIdealGas2D.f90."""

    def __init__(self, mesh, geometry, form=FP64, stream=None, Cp=1.4, Cv=1.0, R=1.0):
        super().__init__(MODEL_CIG, mesh, geometry, form, stream)
        self.SetCv(Cv)
        self.SetCp(Cp)
        self.SetGasConstant(R)

    def SetCp(self, Cp):
        self.Cp = Cp
        self.expansionFactor = Cp / getattr(self, "Cv", 1.0)
        self._push_params()

    def SetCv(self, Cv):
        self.Cv = Cv
        self.expansionFactor = getattr(self, "Cp", 1.4) / Cv
        self._push_params()

    def SetGasConstant(self, R):
        self.R = R
        self._push_params()

    def _environmentals(self):
        if "environmentals" not in self._fields:
            P, nEl = self.N + 1, self.nElem
            self._fields["environmentals"] = torch.zeros((nEl, 2, P, P), device="cuda", dtype=torch.float64)
        return self._fields["environmentals"]

    def SetGravity(self, potential):
        """Gravitational potential -> strong-form gradient (SetGravityFromChar, :604-629)."""
        P, nEl = self.N + 1, self.nElem
        env = self._environmentals()
        env[:, 0].copy_((potential if isinstance(potential, torch.Tensor) else to_device(potential)).reshape(nEl, P, P))
        self._set_field("environmentalsGradient", self._gradient_sf(env, 2))

    def SetDrag(self, Cd):
        env = self._environmentals()
        env[:, 1] = Cd if np.isscalar(Cd) else (Cd if isinstance(Cd, torch.Tensor) else to_device(Cd)).reshape(
            env[:, 1].shape)
        self._set_field("environmentals", env)

    def _pointwise(self, which):
        P, nEl = self.N + 1, self.nElem
        out = torch.zeros((nEl, 4, P, P), device="cuda", dtype=torch.float64)
        if which == "diagnostics":
            lib().CalculateDiagnostics_CompressibleIdealGas2D_gpu_wrapper(
                pp(self.solution.data_ptr()), pp(out.data_ptr()), self.expansionFactor, self.R, self.N, 4, 4, nEl)
        else:
            lib().ConservativeToPrimitive_CompressibleIdealGas2D_gpu_wrapper(
                pp(self.solution.data_ptr()), pp(out.data_ptr()), self.expansionFactor, self.N, 4, nEl)
        return out

    def SetPrescribedSolution(self):
        """Prescribed state from the current solution (:694-743)."""
        prim, diag = self._pointwise("primitive"), self._pointwise("diagnostics")
        self._set_field("prescribedSolution.boundary", self._bnd_interp(self.solution, 4))
        self._set_field("prescribedPrimitive.boundary", self._bnd_interp(prim, 4))
        self._set_field("prescribedDiagnostics.boundary", self._bnd_interp(diag, 4))

    # ---- shock closure (artificial viscosity through BR1)
    def SetClosure(self, mode, c=1.0, s0=None, kappa=1.0, mlp=None):
        """mode CLOSURE_OFF / CLOSURE_INDICATOR / CLOSURE_MLP; nu_e = a c h_e / N max(|u| + c_sound),
        a from the modal-decay indicator (threshold s0 = log10(N^-4) by default, half-width kappa)
        or from the closure MLP (a ClosureMLP, N >= 5)."""
        if mlp is not None:
            w, prm = mlp.device_weights(), mlp.device_params()
            check(lib().selfgpu_model2d_set_mlp(self._h, w.ctypes.data_as(ctypes.c_void_p),
                                                prm.ctypes.data_as(ctypes.c_void_p)))
        if s0 is None:
            s0 = default_s0(self.N)
        self.closure = (mode, c, s0, kappa)
        check(lib().selfgpu_model2d_set_closure(self._h, int(mode), float(c), float(s0), float(kappa),
                                                self.interp.controlPoints.ctypes.data_as(ctypes.c_void_p)))

    def ClosureState(self, reset=False):
        """(nu (nEl,) f64, activation (nEl,) f32, indicator activation (nEl,) f32) of the last
        tendency / RK stage, and (MLP fallbacks, MLP evaluations) since the last reset."""
        nEl = self.nElem
        nu = torch.empty(nEl, device="cuda", dtype=torch.float64)
        act = torch.empty(nEl, device="cuda", dtype=torch.float32)
        ind = torch.empty(nEl, device="cuda", dtype=torch.float32)
        counts = (ctypes.c_int * 2)()
        torch.cuda.synchronize()
        check(lib().selfgpu_model2d_closure_state(self._h, nu.data_ptr(), act.data_ptr(), ind.data_ptr(), counts,
                                                  int(reset)))
        return nu, act, ind, (counts[0], counts[1])

