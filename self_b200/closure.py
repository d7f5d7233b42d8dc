"""Learned shock closure for CompressibleIdealGas2D: the closure MLP, its
training data and its training, on the library's kernels.

The closure replaces the modal-decay indicator's activation a in
nu_e = a c h_e / N max(|u| + c_sound) by a small per-element MLP
(36 -> 32 -> 32 -> 1, ReLU, bfloat16 weights, float32 accumulation, output
clamped to [0, 1]).  Its inputs are the 36 modal-energy features of the
density and the total energy (see ``selfgpu_cig2d_closure_features``); its
training labels are the indicator's activations on states the FP64 method
itself generates; the indicator stays the fallback for features outside the
training range and the judge of the MLP's agreement.

Training data (``harvest``): FP64 runs of seeded four-quadrant 2-D Riemann
problems with the indicator closure on; element states are sampled at several
times, optionally interpolated to a lower degree first (GridInterp with the
Lagrange interpolation matrix between the two Gauss node sets).
"""
import ctypes

import numpy as np
import torch

from . import api as A
from ._lib import check, lib, pp

N_IN, N_HIDDEN = 36, 32
N_MASTER = N_HIDDEN * N_IN + N_HIDDEN + N_HIDDEN * N_HIDDEN + N_HIDDEN + N_HIDDEN + 1  # 2273


def _vp(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def bf16_bits(x):
    """float32 -> bfloat16 bit patterns, round to nearest even."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return b.astype(np.uint16)


class ClosureMLP:
    """Float32 master parameters W1 (32x36), b1, W2 (32x32), b2, w3 (32), b3 and
    the feature range (fmin, fmax) seen in training."""

    def __init__(self, seed=0, params=None):
        if params is None:
            rng = np.random.Generator(np.random.PCG64(seed))
            W1 = rng.uniform(-1, 1, (N_HIDDEN, N_IN)) * np.sqrt(6.0 / N_IN)
            W2 = rng.uniform(-1, 1, (N_HIDDEN, N_HIDDEN)) * np.sqrt(6.0 / N_HIDDEN)
            w3 = rng.uniform(-1, 1, N_HIDDEN) * np.sqrt(3.0 / N_HIDDEN)
            params = np.concatenate([W1.ravel(), np.full(N_HIDDEN, 0.01), W2.ravel(), np.full(N_HIDDEN, 0.01),
                                     w3, [0.0]])
        self.params = np.ascontiguousarray(params, dtype=np.float32)
        assert self.params.size == N_MASTER
        self.fmin = np.full(N_IN, -1e30, dtype=np.float32)
        self.fmax = np.full(N_IN, 1e30, dtype=np.float32)

    # parameter views
    def unpack(self):
        p, o = self.params, 0
        W1 = p[o:o + N_HIDDEN * N_IN].reshape(N_HIDDEN, N_IN); o += N_HIDDEN * N_IN
        b1 = p[o:o + N_HIDDEN]; o += N_HIDDEN
        W2 = p[o:o + N_HIDDEN * N_HIDDEN].reshape(N_HIDDEN, N_HIDDEN); o += N_HIDDEN * N_HIDDEN
        b2 = p[o:o + N_HIDDEN]; o += N_HIDDEN
        w3 = p[o:o + N_HIDDEN]; o += N_HIDDEN
        return W1, b1, W2, b2, w3, float(p[o])

    def device_weights(self):
        W1, _, W2, _, w3, _ = self.unpack()
        return np.ascontiguousarray(bf16_bits(np.concatenate([W1.ravel(), W2.ravel(), w3])))

    def device_params(self):
        _, b1, _, b2, _, b3 = self.unpack()
        return np.ascontiguousarray(np.concatenate([b1, b2, [b3], self.fmin, self.fmax]).astype(np.float32))

    def train(self, features, labels, epochs=20, batch=4096, lr=2e-3, seed=1, stream=None):
        """features: device float32 (n, 36) (feature index fastest); labels: device float32 (n,).
        Returns the per-epoch mean squared error."""
        assert features.is_cuda and features.dtype == torch.float32 and features.shape[1] == N_IN
        n = features.shape[0]
        f = features.contiguous()
        y = labels.contiguous().to(torch.float32)
        self.fmin = f.min(dim=0).values.cpu().numpy().astype(np.float32)
        self.fmax = f.max(dim=0).values.cpu().numpy().astype(np.float32)
        loss = np.zeros(epochs, dtype=np.float32)
        torch.cuda.synchronize()
        check(lib().selfgpu_mlp_train(f.data_ptr(), y.data_ptr(), int(n), int(epochs), int(batch), float(lr),
                                      int(seed), _vp(self.params), _vp(loss), stream))
        return loss

    def infer(self, features, stream=None):
        f = features.contiguous()
        out = torch.empty(f.shape[0], device=f.device, dtype=torch.float32)
        torch.cuda.synchronize()
        check(lib().selfgpu_mlp_infer(f.data_ptr(), int(f.shape[0]), _vp(self.device_weights()),
                                      _vp(self.device_params()), out.data_ptr(), stream))
        return out

    def save(self, path):
        np.savez(path, params=self.params, fmin=self.fmin, fmax=self.fmax)

    @classmethod
    def load(cls, path):
        d = np.load(path)
        m = cls(params=d["params"])
        m.fmin, m.fmax = d["fmin"].astype(np.float32), d["fmax"].astype(np.float32)
        return m


def features(solution, interp, s0=None, kappa=1.0, stream=None):
    """Indicator activation (nEl,) and features (nEl, 36) of a device CIG state
    (nEl, 4, P, P) FP64, float32 device tensors."""
    N = interp.N
    nEl = solution.shape[0]
    act = torch.empty(nEl, device="cuda", dtype=torch.float32)
    feat = torch.empty((nEl, N_IN), device="cuda", dtype=torch.float32) if N >= 5 else None
    torch.cuda.synchronize()
    check(lib().selfgpu_cig2d_closure_features(solution.data_ptr(), N, nEl, _vp(interp.controlPoints),
                                               _vp(interp.qWeights), float(A.default_s0(N) if s0 is None else s0),
                                               float(kappa), act.data_ptr(),
                                               feat.data_ptr() if feat is not None else None, stream))
    torch.cuda.synchronize()
    return act, feat


def grid_interp(solution, N_from, N_to, nVar=4):
    """Interpolate (nEl, nVar, P, P) from the degree-N_from Gauss nodes to the
    degree-N_to Gauss nodes (ScalarGridInterp_2D with the Lagrange iMatrix)."""
    L = A.Lagrange(N_from, A.GAUSS, N_to, A.GAUSS)
    nEl = solution.shape[0]
    out = torch.empty((nEl, nVar, N_to + 1, N_to + 1), device="cuda", dtype=torch.float64)
    lib().ScalarGridInterp_2D_gpu_wrapper(pp(L.device("iMatrix").data_ptr()), pp(solution.data_ptr()),
                                          pp(out.data_ptr()), N_from, N_to, nVar, nEl)
    torch.cuda.synchronize()
    return out


def riemann_quadrants(x, rng, gamma=1.4, rho=(0.1, 1.5), p=(0.1, 1.5), umax=1.0, center=(0.3, 0.7)):
    """Seeded four-quadrant 2-D Riemann state on node coordinates x
    (nEl, 1, P, P, 2): quadrant states (rho, u, v, p) with rho, p uniform in the
    given ranges and |u| <= umax, split at a random centre.  Returns (nEl, 4, P, P)
    conservative (rho u, rho v, rho, rho E)."""
    X, Y = x[:, 0, :, :, 0], x[:, 0, :, :, 1]
    xc, yc = rng.uniform(*center, size=2)
    q = torch.empty((X.shape[0], 4) + tuple(X.shape[1:]), device=X.device, dtype=torch.float64)
    quad = (X >= xc).to(torch.int64) + 2 * (Y >= yc).to(torch.int64)
    r_, u_, v_, p_ = [torch.empty_like(X) for _ in range(4)]
    for k in range(4):
        m = quad == k
        sp = rng.uniform(0.0, umax)
        ang = rng.uniform(0.0, 2.0 * np.pi)
        r_[m], p_[m] = float(rng.uniform(*rho)), float(rng.uniform(*p))
        u_[m], v_[m] = float(sp * np.cos(ang)), float(sp * np.sin(ang))
    q[:, 0], q[:, 1], q[:, 2] = r_ * u_, r_ * v_, r_
    q[:, 3] = p_ / (gamma - 1.0) + 0.5 * r_ * (u_ * u_ + v_ * v_)
    return q


def shock_band(x, rng, gamma=1.4):
    """Smooth density wave (rho = 1 + 0.1 sin(2 pi x) sin(2 pi y), (u, v) =
    (0.5, 0.3), p = 1) plus one seeded shock-tube band: in |y - y0| < 0.05 a
    Sod-like tube (rho, p) = (1, 1) | (0.125, 0.1) at rest, split at x = x0.
    x: node coordinates (nEl, 1, P, P, 2); returns (nEl, 4, P, P) conservative."""
    X, Y = x[:, 0, :, :, 0], x[:, 0, :, :, 1]
    x0, y0 = rng.uniform(0.3, 0.7, size=2)
    rho = 1.0 + 0.1 * torch.sin(2 * np.pi * X) * torch.sin(2 * np.pi * Y)
    u = torch.full_like(X, 0.5)
    v = torch.full_like(X, 0.3)
    p = torch.ones_like(X)
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


def stable_dt(model, q, c_av=1.0, cfl=0.5, cfl_visc=0.25, gamma=1.4):
    """Time step for the closure run: min of the advective CFL step and the
    explicit viscous limit with the largest viscosity the closure can give."""
    rho = q[:, 2]
    u, v = q[:, 0] / rho, q[:, 1] / rho
    pr = (gamma - 1.0) * (q[:, 3] - 0.5 * rho * (u * u + v * v))
    lam = float((torch.sqrt(u * u + v * v) + torch.sqrt(gamma * pr / rho)).max())
    arc = model.geometry.CovariantArcMin()
    h = float(model._wJ().sum(dim=(1, 2)).sqrt().max()) if hasattr(model, "_wJ") else arc
    nu_max = c_av * h / model.N * lam
    dt_adv = cfl * arc / lam
    dt_vis = cfl_visc * arc * arc / max(nu_max, 1e-300)
    return min(dt_adv, dt_vis)


def harvest(N_run, nx, n_problems, snapshots, steps_between, seed=0, N_sample=None, c_av=1.0, stream=None):
    """Features and indicator labels from FP64 indicator-closure runs of seeded
    four-quadrant Riemann problems on a periodic nx x nx mesh at degree N_run,
    sampled every steps_between RK3 steps (snapshots times per problem), the
    states interpolated to each sample degree first when it differs from
    N_run.  N_sample is one degree (returns float32 device tensors (n, 36),
    (n,)) or a tuple of degrees (returns {degree: (features, labels)})."""
    degrees = (N_run,) if N_sample is None else (N_sample if isinstance(N_sample, (tuple, list)) else (N_sample,))
    rng = np.random.Generator(np.random.PCG64(seed))
    interp = A.Lagrange(N_run, A.GAUSS, N_run, A.UNIFORM)
    mesh = A.Mesh2D(nx, nx, periodic=(True, True))
    geo = A.SEMQuad(interp, mesh)
    samp = {d: A.Lagrange(d, A.GAUSS, d, A.UNIFORM) for d in degrees}
    out = {d: ([], []) for d in degrees}
    for _ in range(n_problems):
        model = A.CompressibleIdealGas2D(mesh, geo, form=A.FP64, stream=stream)
        q0 = riemann_quadrants(geo.x, rng)
        model.SetSolution(q0)
        model.SetClosure(A.CLOSURE_INDICATOR, c=c_av)
        dt = stable_dt(model, q0, c_av=c_av)
        for s in range(snapshots):
            if s > 0:
                model.ForwardStep(steps_between, dt)
                model.Sync()
            for d in degrees:
                state = model.solution if d == N_run else grid_interp(model.solution, N_run, d)
                act, feat = features(state, samp[d])
                out[d][0].append(feat)
                out[d][1].append(act)
        model.CheckFinite()
        del model
    res = {d: (torch.cat(f), torch.cat(l)) for d, (f, l) in out.items()}
    if isinstance(N_sample, (tuple, list)):
        return res
    return res[degrees[0]]
