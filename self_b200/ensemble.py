"""Batched ensembles of independent 2-D instances (ShallowWater and
CompressibleIdealGas2D).

An ensemble is many small, unevenly sized 2-D problems advanced together.
Instances of the same degree N are concatenated into one element set: their
sideInfo neighbour ids are offset so that no face crosses an instance, and
each element carries its instance's own time step ("elementDt"), so one fused
launch per RK stage advances every instance of that degree.  The per-degree
handles run on their own streams, each replaying a captured RK step, and the
autotuner picks each handle's kernel variant and consumer-group count.

ShallowWater instances follow the ensemble workload: mesh sizes nx, ny ~
U{8..64}, N ~ U{3, 5, 7}, reflecting walls, g = 1, f = 0, topography h = 1 -
sum of 4 Gaussians (height 0.05..0.2, width 0.05..0.2), fluid thickness H =
h + A exp(-|x - c|^2 / 0.1^2) with A ~ U[1e-3, 1e-2], Hu = Hv = 0, and a
CFL-0.5 time step per instance from CovariantArcMin.

CompressibleIdealGas2D instances (the batched form of the learned-closure
solve): periodic meshes nx, ny ~ U{8..64} with nodes perturbed by 0.02 h,
N ~ U{5, 7}, a smooth density wave with a seeded wavenumber, amplitude and
constant velocity, and in a seeded quarter of the instances one shock-tube
band as well; the shock closure (indicator or MLP) runs over the concatenated
element set, its viscosity and gradient per element, so instances stay
independent.
"""
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import api as A
from ._lib import check, lib


@dataclass
class Instance:
    nx: int
    ny: int
    N: int
    bumps: np.ndarray = field(repr=False)  # (4, 4): height, width, cx, cy
    wave: np.ndarray = field(repr=False)   # (3,): amplitude, cx, cy
    dt: float = 0.0
    group: int = -1
    offset: int = 0

    @property
    def nElem(self):
        return self.nx * self.ny

    def dof(self):
        return 3 * (self.N + 1) ** 2 * self.nElem


def make_instances(n=256, seed=0, nmin=8, nmax=64, degrees=(3, 5, 7)):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        nx, ny = (int(v) for v in rng.integers(nmin, nmax + 1, size=2))
        N = int(rng.choice(degrees))
        bumps = np.stack([rng.uniform(0.05, 0.2, 4), rng.uniform(0.05, 0.2, 4), rng.uniform(0, 1, 4),
                          rng.uniform(0, 1, 4)], axis=1)
        wave = np.array([rng.uniform(1e-3, 1e-2), rng.uniform(0.2, 0.8), rng.uniform(0.2, 0.8)])
        out.append(Instance(nx, ny, N, bumps, wave))
    return out


def topography(inst, X, Y, xp=np):
    h = 1.0
    for a, s, cx, cy in inst.bumps:
        h = h - a * xp.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (s * s))
    return h


def thickness(inst, X, Y, xp=np):
    A_, cx, cy = inst.wave
    return topography(inst, X, Y, xp) + A_ * xp.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / 0.01)


def concat_meshes(meshes):
    """One Mesh2D holding the given meshes' elements one after another (their
    neighbour ids offset), and each mesh's first element in it."""
    coords, sides, offs, off = [], [], [], 0
    for m in meshes:
        si = m.sideInfo.copy(order="F")
        nb = si[2] > 0
        si[2][nb] += off
        coords.append(m.nodeCoords)
        sides.append(si)
        offs.append(off)
        off += m.nElem
    return A.Mesh2D.from_arrays(np.concatenate(coords, axis=3), np.concatenate(sides, axis=2)), offs


def arc_lengths(geo, N):
    """Per-node CovariantArcMin terms 2 min(|dx/ds|, |dx/dt|) / N^2, (nEl, P, P)."""
    d = geo.dxds[:, 0]
    return 2.0 * torch.minimum(torch.sqrt(d[..., 0, 0] ** 2 + d[..., 1, 0] ** 2),
                               torch.sqrt(d[..., 0, 1] ** 2 + d[..., 1, 1] ** 2)) / float(N * N)


class _Ensemble:
    """Instances grouped by degree; one fused handle per degree on its own
    stream.  ForwardStep advances every handle with one CUDA graph launch per
    RK step (selfgpu_ensemble_rk3: one graph branch per degree, so the
    degrees' kernels run concurrently), or, with one_graph=False, each handle
    replays its own captured step on its stream.  Subclasses build a group's
    model (_build_group)."""

    def __init__(self, instances, form, autotune, shared_stream=False, one_graph=True):
        self.instances, self.form = instances, form
        self.groups = {}
        for inst in instances:
            self.groups.setdefault(inst.N, []).append(inst)
        self.handles = {}
        one = torch.cuda.Stream() if shared_stream else None
        for gi, (N, members) in enumerate(sorted(self.groups.items())):
            mesh, offs = concat_meshes([self._instance_mesh(i) for i in members])
            for inst, off in zip(members, offs):
                inst.offset, inst.group = off, gi
            stream = one if one is not None else torch.cuda.Stream()
            h = self._build_group(N, members, mesh, stream)
            h.update(stream=stream, mesh=mesh, members=members)
            h["q0"] = h["model"].solution.clone()
            torch.cuda.synchronize()
            self.handles[N] = h
        self.one_graph = one_graph
        self._ens = None
        self.tuning = {}
        if autotune:
            for N, h in self.handles.items():
                p, c, us = A.ctypes.c_int(), A.ctypes.c_int(), A.ctypes.c_float()
                check(lib().selfgpu_model2d_autotune(h["model"]._h, A.ctypes.byref(p), A.ctypes.byref(c),
                                                     A.ctypes.byref(us)))
                self.tuning[N] = {"persistent": p.value, "groups": c.value, "us_per_stage": us.value}

    def reset(self):
        for h in self.handles.values():
            with torch.cuda.stream(h["stream"]):
                h["model"].SetSolution(h["q0"])
                h["model"].workSol.zero_()
        torch.cuda.synchronize()

    def _ensemble(self):
        if self._ens is None:
            hs = [h["model"]._h for h in self.handles.values()]
            arr = (A.ctypes.c_void_p * len(hs))(*hs)
            out = A.ctypes.c_void_p()
            check(lib().selfgpu_ensemble_create(arr, len(hs), None, A.ctypes.byref(out)))
            self._ens = out
        return self._ens

    def close(self):
        if getattr(self, "_ens", None) is not None:
            lib().selfgpu_ensemble_destroy(self._ens)
            self._ens = None

    def __del__(self):
        self.close()

    def ForwardStep(self, nSteps):
        """nSteps RK3 steps of every instance (each with its own dt), the
        per-degree handles' kernels running concurrently."""
        if self.one_graph:
            check(lib().selfgpu_ensemble_rk3(self._ensemble(), 0.0, int(nSteps)))
            return
        for h in self.handles.values():
            with torch.cuda.stream(h["stream"]):
                check(lib().selfgpu_model2d_rk3(h["model"]._h, 0.0, int(nSteps)))

    def solution(self, inst):
        h = self.handles[inst.N]
        return h["model"].solution[inst.offset:inst.offset + inst.nElem]

    def dof(self):
        return sum(i.dof() for i in self.instances)

    def launches(self):
        return sum(lib().selfgpu_model2d_launch_count(h["model"]._h) for h in self.handles.values())


class ShallowWaterEnsemble(_Ensemble):
    """Batched ShallowWater instances."""

    def __init__(self, instances, form=A.FP32_BULK, cfl=0.5, autotune=True, g=1.0, shared_stream=False,
                 one_graph=True):
        self.cfl, self.g = cfl, g
        super().__init__(instances, form, autotune, shared_stream, one_graph)

    @staticmethod
    def _instance_mesh(inst):
        return A.Mesh2D(inst.nx, inst.ny, bcid=A.BC_NONORMALFLOW)

    def _build_group(self, N, members, mesh, stream):
        interp = A.Lagrange(N)
        geo = A.SEMQuad(interp, mesh)
        model = A.ShallowWater(mesh, geo, form=self.form, stream=stream.cuda_stream)
        model.g = self.g
        model._push_params()
        X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]  # (nEl, P, P)
        P = N + 1
        h = torch.empty_like(X)
        H = torch.empty_like(X)
        for inst in members:
            sl = slice(inst.offset, inst.offset + inst.nElem)
            h[sl] = topography(inst, X[sl], Y[sl], xp=torch)
            H[sl] = thickness(inst, X[sl], Y[sl], xp=torch)
        model.SetTopography(h.reshape(-1, 1, P, P))
        q = torch.zeros((mesh.nElem, 3, P, P), device="cuda", dtype=torch.float64)
        q[:, 2] = H
        model.SetSolution(q)
        # CFL time step per instance: cfl * CovariantArcMin / max(|u| + sqrt(g H)), u = 0 at start
        ds = arc_lengths(geo, N)
        dtE = torch.empty(mesh.nElem, device="cuda", dtype=torch.float64)
        for inst in members:
            sl = slice(inst.offset, inst.offset + inst.nElem)
            cmax = float(torch.sqrt(self.g * H[sl].max()))
            inst.dt = self.cfl * float(ds[sl].min()) / cmax
            dtE[sl] = inst.dt
        model._set_field("elementDt", dtE)
        return {"model": model, "geo": geo, "dt": dtE}


class UnbatchedShallowWater:
    """The same instances advanced one handle per instance, sequentially: the
    plain FP64 GPU form an ensemble is compared against."""

    def __init__(self, instances, g=1.0, form=A.FP64):
        self.runs = []
        for inst in instances:
            mesh = A.Mesh2D(inst.nx, inst.ny, bcid=A.BC_NONORMALFLOW)
            geo = A.SEMQuad(A.Lagrange(inst.N), mesh)
            model = A.ShallowWater(mesh, geo, form=form)
            model.g = g
            model._push_params()
            X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]
            P = inst.N + 1
            model.SetTopography(topography(inst, X, Y, xp=torch).reshape(-1, 1, P, P))
            q = torch.zeros((mesh.nElem, 3, P, P), device="cuda", dtype=torch.float64)
            q[:, 2] = thickness(inst, X, Y, xp=torch)
            model.SetSolution(q)
            self.runs.append((inst, model, q.clone()))

    def reset(self):
        for _, model, q0 in self.runs:
            model.SetSolution(q0)
            model.workSol.zero_()
        torch.cuda.synchronize()

    def ForwardStep(self, nSteps):
        for inst, model, _ in self.runs:
            model.ForwardStep(nSteps, inst.dt)

    def launches(self):
        return sum(model.LaunchCount() for _, model, _ in self.runs)


@dataclass
class GasInstance:
    """One CompressibleIdealGas2D instance of the batched learned-closure form."""
    nx: int
    ny: int
    N: int
    wave: np.ndarray = field(repr=False)  # kx, ky, amplitude, u, v
    band: np.ndarray = field(repr=False)  # x0, y0 of a shock-tube band, or empty (smooth instance)
    dt: float = 0.0
    group: int = -1
    offset: int = 0

    @property
    def nElem(self):
        return self.nx * self.ny

    @property
    def smooth(self):
        return self.band.size == 0

    def dof(self):
        return 4 * (self.N + 1) ** 2 * self.nElem


def make_gas_instances(n=256, seed=0, nmin=8, nmax=64, degrees=(5, 7), shock_fraction=0.25):
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(n):
        nx, ny = (int(v) for v in rng.integers(nmin, nmax + 1, size=2))
        N = int(rng.choice(degrees))
        wave = np.array([rng.integers(1, 3), rng.integers(1, 3), rng.uniform(0.05, 0.15), rng.uniform(-0.5, 0.5),
                         rng.uniform(-0.5, 0.5)], dtype=np.float64)
        band = rng.uniform(0.3, 0.7, size=2) if rng.uniform() < shock_fraction else np.zeros(0)
        out.append(GasInstance(nx, ny, N, wave, band))
    return out


def gas_state(inst, X, Y, gamma=1.4):
    """Conservative state (n, 4, P, P) of an instance on node coordinates X, Y
    (n, P, P): rho = 1 + A sin(2 pi kx x) sin(2 pi ky y), constant (u, v), p = 1,
    and for a shocked instance a Sod-like band (rho, p) = (1, 1) | (0.125, 0.1)
    at rest in |y - y0| < 0.05, split at x = x0."""
    kx, ky, amp, u0, v0 = inst.wave
    rho = 1.0 + amp * torch.sin(2 * np.pi * kx * X) * torch.sin(2 * np.pi * ky * Y)
    u = torch.full_like(X, u0)
    v = torch.full_like(X, v0)
    p = torch.ones_like(X)
    if not inst.smooth:
        x0, y0 = inst.band
        band = (Y - y0).abs() < 0.05
        left = X < x0
        rho = torch.where(band, torch.where(left, torch.ones_like(X), torch.full_like(X, 0.125)), rho)
        p = torch.where(band, torch.where(left, torch.ones_like(X), torch.full_like(X, 0.1)), p)
        u = torch.where(band, torch.zeros_like(X), u)
        v = torch.where(band, torch.zeros_like(X), v)
    q = torch.empty((X.shape[0], 4) + tuple(X.shape[1:]), device=X.device, dtype=torch.float64)
    q[:, 0], q[:, 1], q[:, 2] = rho * u, rho * v, rho
    q[:, 3] = p / (gamma - 1.0) + 0.5 * rho * (u * u + v * v)
    return q


def _gas_mesh(inst):
    return A.Mesh2D(inst.nx, inst.ny, periodic=(True, True), perturbation=0.02)


def _gas_dt(q, arc, wJ, N, cfl=0.5, cfl_visc=0.02, c_av=1.0, gamma=1.4):
    """The closure run's time step of one instance: min of the advective CFL
    step and the explicit viscous limit cfl_visc * ArcMin^2 / nu_max with the
    largest viscosity the closure can give.  The viscous factor is far below
    closure.stable_dt's 0.25: on these coarse meshes a shock-tube band lies
    inside single elements, the closure acts at full strength from the first
    step, and the BR1 operator's explicit limit measured with the oracle is
    about a tenth of 0.25 ArcMin^2 / nu_max."""
    rho = q[:, 2]
    u, v = q[:, 0] / rho, q[:, 1] / rho
    pr = (gamma - 1.0) * (q[:, 3] - 0.5 * rho * (u * u + v * v))
    lam = float((torch.sqrt(u * u + v * v) + torch.sqrt(gamma * pr / rho)).max())
    h = float(wJ.sum(dim=(1, 2)).sqrt().max())
    nu_max = c_av * h / N * lam
    return min(cfl * arc / lam, cfl_visc * arc * arc / max(nu_max, 1e-300))


class CompressibleGasEnsemble(_Ensemble):
    """Batched CompressibleIdealGas2D instances with an optional shock closure
    (closure = CLOSURE_OFF / CLOSURE_INDICATOR / CLOSURE_MLP; mlps maps a
    degree to its ClosureMLP)."""

    def __init__(self, instances, form=A.FP32_BULK, closure=A.CLOSURE_OFF, mlps=None, c_av=1.0, autotune=True,
                 one_graph=True):
        self.closure, self.mlps, self.c_av = closure, mlps or {}, c_av
        super().__init__(instances, form, autotune, one_graph=one_graph)

    @staticmethod
    def _instance_mesh(inst):
        return _gas_mesh(inst)

    def _build_group(self, N, members, mesh, stream):
        interp = A.Lagrange(N, A.GAUSS, N, A.UNIFORM)
        geo = A.SEMQuad(interp, mesh)
        model = A.CompressibleIdealGas2D(mesh, geo, form=self.form, stream=stream.cuda_stream)
        X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]
        P = N + 1
        q = torch.empty((mesh.nElem, 4, P, P), device="cuda", dtype=torch.float64)
        for inst in members:
            sl = slice(inst.offset, inst.offset + inst.nElem)
            q[sl] = gas_state(inst, X[sl], Y[sl])
        model.SetSolution(q)
        ds, wJ = arc_lengths(geo, N), model._wJ()
        dtE = torch.empty(mesh.nElem, device="cuda", dtype=torch.float64)
        for inst in members:
            sl = slice(inst.offset, inst.offset + inst.nElem)
            inst.dt = _gas_dt(q[sl], float(ds[sl].min()), wJ[sl], N, c_av=self.c_av)
            dtE[sl] = inst.dt
        model._set_field("elementDt", dtE)
        if self.closure != A.CLOSURE_OFF:
            model.SetClosure(self.closure, c=self.c_av, mlp=self.mlps.get(N) if self.closure == A.CLOSURE_MLP
                             else None)
        return {"model": model, "geo": geo, "dt": dtE}


class UnbatchedGas:
    """The same CompressibleIdealGas2D instances advanced one handle per
    instance, sequentially, in the plain FP64 form (no closure): the form the
    batched learned-closure form is compared against."""

    def __init__(self, instances, form=A.FP64):
        self.runs = []
        for inst in instances:
            mesh = _gas_mesh(inst)
            geo = A.SEMQuad(A.Lagrange(inst.N, A.GAUSS, inst.N, A.UNIFORM), mesh)
            model = A.CompressibleIdealGas2D(mesh, geo, form=form)
            X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]
            q = gas_state(inst, X, Y)
            model.SetSolution(q)
            if inst.dt == 0.0:  # the same step the batched ensemble gives this instance
                inst.dt = _gas_dt(q, float(arc_lengths(geo, inst.N).min()), model._wJ(), inst.N)
            self.runs.append((inst, model, q.clone()))

    def reset(self):
        for _, model, q0 in self.runs:
            model.SetSolution(q0)
            model.workSol.zero_()
        torch.cuda.synchronize()

    def ForwardStep(self, nSteps):
        for inst, model, _ in self.runs:
            model.ForwardStep(nSteps, inst.dt)

    def launches(self):
        return sum(model.LaunchCount() for _, model, _ in self.runs)


def time_it(fn, reps=1):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / reps
