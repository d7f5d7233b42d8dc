"""Batched ensembles of independent ShallowWater instances.

An ensemble is many small, unevenly sized 2-D problems advanced together.
Instances of the same degree N are concatenated into one element set: their
sideInfo neighbour ids are offset so that no face crosses an instance, and
each element carries its instance's own time step ("elementDt"), so one fused
launch per RK stage advances every instance of that degree.  The per-degree
handles run on their own streams, each replaying a captured RK step, and the
autotuner picks each handle's kernel variant and consumer-group count.

The default instance generator follows the ensemble workload: mesh sizes
nx, ny ~ U{8..64}, N ~ U{3, 5, 7}, reflecting walls, g = 1, f = 0, topography
h = 1 - sum of 4 Gaussians (height 0.05..0.2, width 0.05..0.2), fluid
thickness H = h + A exp(-|x - c|^2 / 0.1^2) with A ~ U[1e-3, 1e-2], Hu = Hv = 0,
and a CFL-0.5 time step per instance from CovariantArcMin.
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


class ShallowWaterEnsemble:
    """Instances grouped by degree; one fused handle per degree."""

    def __init__(self, instances, form=A.FP32_BULK, cfl=0.5, autotune=True, g=1.0):
        self.instances, self.form, self.g = instances, form, g
        self.groups = {}
        for inst in instances:
            self.groups.setdefault(inst.N, []).append(inst)
        self.handles = {}
        for gi, (N, members) in enumerate(sorted(self.groups.items())):
            self.handles[N] = self._build_group(N, members, cfl, gi)
        self.tuning = {}
        if autotune:
            for N, h in self.handles.items():
                p, c, us = A.ctypes.c_int(), A.ctypes.c_int(), A.ctypes.c_float()
                check(lib().selfgpu_model2d_autotune(h["model"]._h, A.ctypes.byref(p), A.ctypes.byref(c),
                                                     A.ctypes.byref(us)))
                self.tuning[N] = {"persistent": p.value, "groups": c.value, "us_per_stage": us.value}

    def _build_group(self, N, members, cfl, gi):
        # concatenated mesh
        coords, sides, off = [], [], 0
        for inst in members:
            m = A.Mesh2D(inst.nx, inst.ny, bcid=A.BC_NONORMALFLOW)
            si = m.sideInfo.copy(order="F")
            nb = si[2] > 0
            si[2][nb] += off
            coords.append(m.nodeCoords)
            sides.append(si)
            inst.offset, inst.group = off, gi
            off += m.nElem
        mesh = A.Mesh2D.from_arrays(np.concatenate(coords, axis=3), np.concatenate(sides, axis=2))
        interp = A.Lagrange(N)
        geo = A.SEMQuad(interp, mesh)
        stream = torch.cuda.Stream()
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
        d = geo.dxds[:, 0]
        ds = 2.0 * torch.minimum(torch.sqrt(d[..., 0, 0] ** 2 + d[..., 1, 0] ** 2),
                                 torch.sqrt(d[..., 0, 1] ** 2 + d[..., 1, 1] ** 2)) / float(N * N)
        dtE = torch.empty(mesh.nElem, device="cuda", dtype=torch.float64)
        for inst in members:
            sl = slice(inst.offset, inst.offset + inst.nElem)
            cmax = float(torch.sqrt(self.g * H[sl].max()))
            inst.dt = cfl * float(ds[sl].min()) / cmax
            dtE[sl] = inst.dt
        model._set_field("elementDt", dtE)
        torch.cuda.synchronize()
        return {"model": model, "stream": stream, "mesh": mesh, "geo": geo, "members": members, "dt": dtE,
                "q0": q.clone()}

    def reset(self):
        for h in self.handles.values():
            with torch.cuda.stream(h["stream"]):
                h["model"].SetSolution(h["q0"])
                h["model"].workSol.zero_()
        torch.cuda.synchronize()

    def ForwardStep(self, nSteps):
        """nSteps RK3 steps of every instance (each with its own dt); the
        per-degree handles run concurrently on their streams."""
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


def time_it(fn, reps=1):
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        fn()
    torch.cuda.synchronize()
    return (time.perf_counter() - t0) / reps
