"""The zero-allocation CompressibleIdealGas2D tendency entry point.

selfgpu_cig2d_tendency_noalloc serves callers that may not allocate device
memory when they need a tendency (all device memory owned by the host code, a
hard memory cap, no allocator calls allowed inside a solver step).  Its
scratch is a fixed device array inside the library.  These tests call it
through the C ABI twice in a row, on two different states, and check each
result against the engine's selfgpu_model2d_tendency on the same inputs: bit
for bit against the reference-rounding form (SELFGPU_FP64_REF, the same
arithmetic) and within the 1e-12 relative tolerance of the other parity tests
against the production FP64 form.  They also check the fixed-size limit at
N = 3 from both sides and the refusal of boundary conditions it cannot serve.

This file is collected last so that a run stopping at the first failure has
run every other test before it.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-12
SCRATCH_BYTES = 16 * 1024 * 1024  # SELFGPU_NOALLOC_SCRATCH_BYTES


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


def _limit(N):
    """Largest element count the fixed scratch takes at degree N."""
    block = (9 * (N + 1) + 1) // 2 * 2  # values per (element, side) trace block
    return SCRATCH_BYTES // (4 * block * 8)


def _call(S, q, out, geo, mesh, interp, gamma):
    L = S.lib()
    dg = np.asfortranarray(interp.dgMatrix)
    bm = np.asfortranarray(interp.bMatrix)
    qw = np.asfortranarray(interp.qWeights)
    si_h = np.asfortranarray(mesh.sideInfo)
    host = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    dev = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    return L.selfgpu_cig2d_tendency_noalloc(dev(q), dev(out), dev(geo.dsdx), dev(geo.J), dev(geo.nHat),
                                            dev(geo.nScale), dev(mesh.sideInfo_d), host(si_h), host(dg),
                                            host(bm), host(qw), gamma, interp.N, mesh.nElem, None)


def _check_two_calls(S, mesh, N):
    interp = S.Lagrange(N)
    geo = S.SEMQuad(interp, mesh)
    ref_model = S.CompressibleIdealGas2D(mesh, geo, form=S.FP64_REF)
    prod_model = S.CompressibleIdealGas2D(mesh, geo, form=S.FP64)
    for seed in (1, 2):  # two calls in a row, on different states
        q = _state(geo.x, seed)
        ref_model.SetSolution(q)
        ref = ref_model.CalculateTendency().clone()
        prod_model.SetSolution(q)
        prod = prod_model.CalculateTendency().clone()
        out = torch.full_like(ref, float("nan"))
        rc = _call(S, q, out, geo, mesh, interp, ref_model.expansionFactor)
        assert rc == 0, S.lib().selfgpu_last_error()
        torch.cuda.synchronize()
        assert torch.isfinite(out).all()
        assert torch.equal(out, ref)
        assert _rel(out, prod) < TOL


# N = 1 is left out: the reference's LegendreGauss fills the second Gauss node
# of N = 1 from its output arrays instead of the computed first node
# (src/SELF_Quadrature.f90:217-222), so with zeroed arrays that quadrature has
# a zero weight and every N = 1 Gauss model divides by it (the oracle too).
@pytest.mark.parametrize("N", [2, 3, 5, 7])
def test_noalloc_tendency_matches_engine_on_two_calls_in_a_row(N):
    import self_b200 as S
    mesh = S.Mesh2D(6, 5, periodic=(True, False), perturbation=0.04, bcid=S.BC_NONORMALFLOW,
                    rotation=[0, 1, 2, 3, 0] * 6)
    _check_two_calls(S, mesh, N)


def test_noalloc_at_the_element_limit_at_n3():
    """The largest mesh the fixed scratch takes at N = 3 (one row of elements,
    walls all round) runs and matches the engine; one element more is
    refused."""
    import self_b200 as S
    N = 3
    n = _limit(N)
    assert n == 14563
    _check_two_calls(S, S.Mesh2D(n, 1, bcid=S.BC_NONORMALFLOW), N)
    big = S.Mesh2D(n + 1, 1, bcid=S.BC_NONORMALFLOW)
    interp = S.Lagrange(N)
    geo = S.SEMQuad(interp, big)
    q = torch.zeros((big.nElem, 4, N + 1, N + 1), device="cuda", dtype=torch.float64)
    rc = _call(S, q, q.clone(), geo, big, interp, 1.4)
    assert rc == 1
    assert b"fixed limit" in S.lib().selfgpu_last_error()


def test_noalloc_rejects_boundary_conditions_it_cannot_serve():
    import self_b200 as S
    N = 3
    for bc in (S.BC_PRESCRIBED, S.BC_RADIATION):
        mesh = S.Mesh2D(3, 3, bcid=bc)
        interp = S.Lagrange(N)
        geo = S.SEMQuad(interp, mesh)
        q = torch.ones((mesh.nElem, 4, N + 1, N + 1), device="cuda", dtype=torch.float64)
        rc = _call(S, q, q.clone(), geo, mesh, interp, 1.4)
        assert rc == 1
        assert b"NONORMALFLOW" in S.lib().selfgpu_last_error()


def test_noalloc_rejects_meshes_beyond_its_fixed_scratch():
    import self_b200 as S
    L = S.lib()
    buf = torch.zeros(64, device="cuda", dtype=torch.float64)
    si = np.zeros(20, dtype=np.int32)
    d = ctypes.c_void_p(buf.data_ptr())
    h = si.ctypes.data_as(ctypes.c_void_p)
    too_many = _limit(7) + 1  # 7282 elements at N = 7 need more than the 16 MiB of face-trace scratch
    rc = L.selfgpu_cig2d_tendency_noalloc(d, d, d, d, d, d, d, h, h, h, h, 1.4, 7, too_many, None)
    assert rc == 1
    assert b"fixed limit" in L.selfgpu_last_error()
