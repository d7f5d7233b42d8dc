"""The reference's own CompressibleIdealGas2D test scenarios run through the
engine in every arithmetic form, against the oracle and against their exact
answer (a state that does not move):

  test/CompressibleIdealGas2D_StaticFluid.f90            fluid at rest, prescribed sides
  test/CompressibleIdealGas2D_StaticFluid_NoNormalFlow.f90  fluid at rest, walls
  test/CompressibleIdealGas2D_ConstantVelocity.f90       uniform flow, prescribed sides

on the Block2D mesh (etc/mesh/Block2D: 5 x 5 elements on the unit square) at
the CLI defaults (N = 7, Gauss nodes, dt = 5e-4, end time 0.01 = 20 steps).
The reference itself asserts only a finite entropy.  Tolerances: 1e-12
relative to the state for both FP64 forms (the reference-rounding form equals
the oracle bit for bit), 1e-6 for the FP32-bulk form.
"""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

N, P, STEPS, DT = 7, 8, 20, 5e-4
SCENARIOS = {"static_prescribed": (O.BC_PRESCRIBED, 0.0, 0.0),
             "static_walls": (O.BC_NONORMALFLOW, 0.0, 0.0),
             "constant_velocity": (O.BC_PRESCRIBED, 0.5, 0.25)}


def _state(nEl, u, v):
    q = np.zeros((P, P, 4, nEl), order="F")
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = u, v, 1.0
    q[:, :, 3] = 1.0 / 0.4 + 0.5 * (u * u + v * v)  # p = 1, gamma = 1.4
    return q


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("scenario", sorted(SCENARIOS))
def test_cig_reference_scenario(scenario, form):
    import self_b200 as S
    bc, u, v = SCENARIOS[scenario]
    om = O.Mesh(5, 5, bcid=bc)
    mod_o = O.Model(O.CIG, N, om)
    q0 = _state(om.nEl, u, v)
    mod_o.set("solution", q0)
    if bc == O.BC_PRESCRIBED:
        mod_o.set("prescribed")
    mod_o.rk3(STEPS, DT)
    want = mod_o.get("solution", q0.shape)

    mesh = S.Mesh2D(5, 5, bcid=bc)
    geo = S.SEMQuad(S.Lagrange(N), mesh)
    mod = S.CompressibleIdealGas2D(mesh, geo, form=form)
    mod.SetSolution(q0)
    if bc == O.BC_PRESCRIBED:
        mod.SetPrescribedSolution()
    mod.ForwardStep(STEPS, DT)
    mod.Sync()
    mod.CheckFinite()
    got = S.to_host(mod.solution).reshape(q0.shape, order="F")
    scale = np.abs(q0).max()
    tol = 1e-6 if form == S.FP32_BULK else 1e-12
    assert np.abs(got - want).max() <= tol * scale, "against the oracle"
    assert np.abs(got - q0).max() <= tol * scale, "against the exact (unchanged) state"
    if form == S.FP64_REF:
        assert np.array_equal(got, want)


@pytest.mark.parametrize("form", [0, 1, 2])
@pytest.mark.parametrize("wave", ["planetary", "topographic"])
def test_lsw_rossby_wave_scenario(wave, form):
    """test/LinearShallowWater2D_PlanetaryRossbyWave.f90 and
    LinearShallowWater2D_TopographicRossbyWave.f90 on GeophysicalBlock2DMedium
    (10 x 10 elements on [-5e5, 5e5]^2), g = 10, radiation sides, N = 7: 20 RK3
    steps of 2 s, against the oracle (per field, relative to the field's
    largest value; the FP32-bulk form to 1e-6 in relative L2 over the state)
    and the entropy not growing."""
    import self_b200 as S
    N, P = 7, 8
    om = O.Mesh(10, 10, -5e5, 5e5, -5e5, 5e5, bcid=O.BC_RADIATION)
    x = O.Geometry(N, om).x
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    f = np.asfortranarray((1e-4 + (2e-11 * Y if wave == "planetary" else 0 * Y)).reshape(P, P, 1, -1, order="F"))
    H = np.asfortranarray((1000.0 + (2e-4 * Y if wave == "topographic" else 0 * Y)).reshape(P, P, 1, -1, order="F"))
    q0 = np.zeros((P, P, 3, om.nEl), order="F")
    q0[:, :, 2] = 1e-2 * np.exp(-(X ** 2 + Y ** 2) / 2e10)
    mod_o = O.Model(O.LSW, N, om, g=10.0)
    mod_o.set("H", H)
    mod_o.set("fCori", f)
    mod_o.set("solution", q0)
    mod_o.rk3(20, 2.0)
    want = mod_o.get("solution", q0.shape)

    mesh = S.Mesh2D(10, 10, -5e5, 5e5, -5e5, 5e5, bcid=S.BC_RADIATION)
    geo = S.SEMQuad(S.Lagrange(N), mesh)
    mod = S.LinearShallowWater(mesh, geo, form=form)
    mod.g = 10.0
    mod.SetBathymetry(H)
    mod.SetCoriolis(f)
    mod.SetSolution(q0)
    e0 = mod.CalculateEntropy()
    mod.ForwardStep(20, 2.0)
    mod.Sync()
    mod.CheckFinite()
    got = S.to_host(mod.solution).reshape(q0.shape, order="F")
    if form == S.FP32_BULK:
        assert np.linalg.norm(got - want) <= 1e-6 * np.linalg.norm(want)
    else:
        for v in range(3):
            scale = np.abs(want[:, :, v]).max()
            assert np.abs(got[:, :, v] - want[:, :, v]).max() <= 1e-12 * scale, v
    if form == S.FP64_REF:
        assert np.array_equal(got, want)
    e1 = mod.CalculateEntropy()
    assert np.isfinite(e1) and e1 <= e0 * (1 + 1e-12)
