"""The zero-allocation CompressibleIdealGas2D tendency entry point.

selfgpu_cig2d_tendency_noalloc serves callers that may not allocate device
memory when they need a tendency (all device memory owned by the host code, a
hard memory cap, no allocator calls allowed inside a solver step).  Its
scratch is a fixed device array inside the library.  This test calls it
through the C ABI twice in a row, on two different states, and checks each
result against the engine's selfgpu_model2d_tendency on the same inputs, with
the 1e-12 relative tolerance of the other parity tests.  It also checks that a
mesh too large for the fixed array is refused with a clear error.

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _state(x, seed):
    rng = np.random.default_rng(seed)
    X, Y = x[..., 0], x[..., 1]  # (nEl, 1, P, P)
    a, b = rng.uniform(0.5, 1.5, 2)
    rho = 1.0 + 0.1 * torch.sin(2 * np.pi * a * X) * torch.sin(2 * np.pi * b * Y)
    u = 0.5 + 0.05 * torch.cos(2 * np.pi * Y)
    v = 0.3 + 0.05 * torch.sin(2 * np.pi * X)
    p = 1.0 + 0.05 * torch.cos(2 * np.pi * (X + Y))
    q = torch.stack([rho * u, rho * v, rho, p / 0.4 + 0.5 * rho * (u * u + v * v)], dim=1)[:, :, 0]
    return q.contiguous()


def _rel(got, ref):
    return float((got - ref).abs().max() / ref.abs().max())


def test_noalloc_tendency_matches_engine_on_two_calls_in_a_row():
    import self_b200 as S
    N = 7
    mesh = S.Mesh2D(6, 5, periodic=(True, False), perturbation=0.04, bcid=S.BC_NONORMALFLOW,
                    rotation=[0, 1, 2, 3, 0] * 6)
    interp = S.Lagrange(N)
    geo = S.SEMQuad(interp, mesh)
    model = S.CompressibleIdealGas2D(mesh, geo)
    L = S.lib()
    dg = np.asfortranarray(interp.dgMatrix)
    bm = np.asfortranarray(interp.bMatrix)
    qw = np.asfortranarray(interp.qWeights)
    si_h = np.asfortranarray(mesh.sideInfo)
    host = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    dev = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    for seed in (1, 2):  # two calls in a row, on different states
        q = _state(geo.x, seed)
        model.SetSolution(q)
        ref = model.CalculateTendency().clone()
        out = torch.full_like(ref, float("nan"))
        rc = L.selfgpu_cig2d_tendency_noalloc(dev(q), dev(out), dev(geo.dsdx), dev(geo.J), dev(geo.nHat),
                                              dev(geo.nScale), dev(mesh.sideInfo_d), host(si_h), host(dg),
                                              host(bm), host(qw), model.expansionFactor, N, mesh.nElem, None)
        assert rc == 0, L.selfgpu_last_error()
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert _rel(out, ref) < TOL


def test_noalloc_rejects_meshes_beyond_its_fixed_scratch():
    import self_b200 as S
    L = S.lib()
    buf = torch.zeros(64, device="cuda", dtype=torch.float64)
    si = np.zeros(20, dtype=np.int32)
    d = ctypes.c_void_p(buf.data_ptr())
    h = si.ctypes.data_as(ctypes.c_void_p)
    too_many = 8000  # 8000 elements at N = 7 need 18.4 MB of face-trace scratch
    rc = L.selfgpu_cig2d_tendency_noalloc(d, d, d, d, d, d, d, h, h, h, h, 1.4, 7, too_many, None)
    assert rc == 1
    assert b"fixed limit" in L.selfgpu_last_error()
