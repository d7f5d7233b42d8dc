"""Pins of the CPU oracle (no GPU).

The reference's tests hold no numeric golden vectors for the tendency path, so
the oracle is pinned by (a) fixtures read from the reference's own mesh files,
(b) published quadrature values (numpy's independent Golub-Welsch), (c) the
exact invariants the reference's scenarios rely on -- free-stream
preservation, the lake at rest known answer of
test/ShallowWater2D_QuietFluid.f90:125-130, discrete conservation, energy
non-increase with reflecting walls -- and (d) its own stored regression
outputs.
"""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("N", [2, 4, 5, 6, 7, 8])
def test_gauss_nodes_match_published_values(N):
    x, w = O.quadrature(N, O.GAUSS)
    xr, wr = np.polynomial.legendre.leggauss(N + 1)
    np.testing.assert_allclose(x, xr, atol=2e-16, rtol=0)
    np.testing.assert_allclose(w, wr, atol=2e-15, rtol=0)


def test_gauss_n3_node_order_quirk():
    # The reference's Newton loop (src/SELF_Quadrature.f90:226-250) runs j to
    # (N+1)/2 and mirrors; at N = 3 the interior pair comes out swapped.  The
    # set is still the Gauss set and the mirror x_{N-i} = -x_i still holds.
    x, w = O.quadrature(3, O.GAUSS)
    xr, wr = np.polynomial.legendre.leggauss(4)
    np.testing.assert_allclose(np.sort(x), xr, atol=2e-16)
    assert x[1] > 0 > x[2]
    np.testing.assert_allclose(x[::-1], -x, atol=0)
    np.testing.assert_allclose(w[::-1], w, atol=0)


@pytest.mark.parametrize("N", [2, 3, 4, 7])
def test_gauss_lobatto(N):
    x, w = O.quadrature(N, O.GAUSS_LOBATTO)
    assert x[0] == -1.0 and x[-1] == 1.0
    np.testing.assert_allclose(w.sum(), 2.0, atol=1e-15)
    # exact for degree 2N-1
    for k in range(2 * N):
        exact = (1 - (-1) ** (k + 1)) / (k + 1)
        np.testing.assert_allclose((w * x ** k).sum(), exact, atol=1e-14)


@pytest.mark.parametrize("N", [2, 3, 5, 7])
def test_lagrange_operators_exact_on_polynomials(N):
    L = O.Lagrange(N, O.GAUSS, 2 * N, O.UNIFORM)
    x = L.controlPoints
    for k in range(N + 1):
        f = x ** k
        df = k * x ** (k - 1) if k else 0 * x
        np.testing.assert_allclose(L.dMatrix.T @ f, df, atol=5e-13 * max(1, k * k))
        # boundary matrix: values at -1 and +1
        np.testing.assert_allclose(L.bMatrix[:, 0] @ f, (-1.0) ** k, atol=1e-13)
        np.testing.assert_allclose(L.bMatrix[:, 1] @ f, 1.0, atol=1e-13)
        # interpolation to the uniform target grid
        np.testing.assert_allclose(L.iMatrix.T @ f, L.targetPoints ** k, atol=1e-13)
    # weak-form relation: dgMatrix(a,b) = -D(a,b) w_a / w_b with D(r,c) = dMatrix(c,r)
    w = L.qWeights
    D = L.dMatrix.T  # D[r, c]: derivative at r from node c
    np.testing.assert_allclose(L.dgMatrix, -D * w[:, None] / w[None, :], rtol=1e-15, atol=1e-15)


@pytest.mark.parametrize("name", ["Block2D", "GeophysicalBlock2DMedium"])
def test_structured_mesh_matches_reference_mesh_files(name):
    ref = json.load(open(os.path.join(GOLD, "reference_meshes.json")))[name]
    nx, ny, x0, x1, y0, y1 = ref["structured"]
    m = O.Mesh(nx, ny, x0, x1, y0, y1, bcid=O.BC_NONORMALFLOW)
    nodes = np.array(ref["nodes"])
    for e, corners in enumerate(ref["elements"]):
        # ISM corners are counter-clockwise from south-west = CN1..CN4
        got = [m.nodeCoords[:, 0, 0, e], m.nodeCoords[:, 1, 0, e], m.nodeCoords[:, 1, 1, e], m.nodeCoords[:, 0, 1, e]]
        want = [nodes[c - 1] for c in corners]
        np.testing.assert_array_equal(np.array(got), np.array(want))
        # ISM boundary names are listed South, East, North, West -- SELF's side order
        for s, bname in enumerate(ref["boundary_names"][e]):
            physical = bname != "---"
            assert (m.sideInfo[2, s, e] == 0) == physical
            assert (m.sideInfo[4, s, e] == O.BC_NONORMALFLOW) == physical


def test_mesh_connectivity_and_flips():
    rot = [0, 1, 2, 3, 1, 2, 3, 0, 2, 3, 0, 1]
    m = O.Mesh(4, 3, periodic=(True, False), rot=rot)
    si = m.sideInfo
    flips = 0
    for e in range(12):
        for s in range(4):
            if si[4, s, e] != 0:
                continue
            e2, s2, flip = si[2, s, e] - 1, si[3, s, e] // 10 - 1, si[3, s, e] % 10
            # the neighbour points back
            assert si[2, s2, e2] - 1 == e and si[3, s2, e2] // 10 - 1 == s
            assert si[3, s2, e2] % 10 == flip
            flips += flip
    assert flips > 0
    # unrotated periodic mesh: all flips zero (shared periodic node ids)
    m = O.Mesh(4, 4, periodic=(True, True))
    assert np.all(m.sideInfo[4] == 0) and np.all(m.sideInfo[3] % 10 == 0)


def _cig_state(x, rho_fn, u, v, p, gamma=1.4):
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    rho = rho_fn(X, Y)
    q = np.zeros(X.shape[:2] + (4, X.shape[2]), order="F")
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * u, rho * v, rho
    q[:, :, 3] = p / (gamma - 1) + 0.5 * rho * (u * u + v * v)
    return q


def test_cig_free_stream_preservation_on_perturbed_periodic_mesh():
    m = O.Mesh(6, 6, periodic=(True, True), amp=0.05)
    mod = O.Model(O.CIG, 5, m)
    q = _cig_state(O.Geometry(5, m).x, lambda X, Y: 1.0 + 0 * X, 0.5, 0.3, 1.0)
    mod.set("solution", q)
    d = mod.tendency()
    assert np.abs(d).max() < 1e-10


def test_sw_lake_at_rest_known_answer():
    # test/ShallowWater2D_QuietFluid.f90:125-130: flat bottom, radiation
    # boundaries, |Hu|,|Hv| <= 1000*eps after the run.
    m = O.Mesh(4, 4, bcid=O.BC_RADIATION)
    mod = O.Model(O.SW, 4, m)
    q = np.zeros((5, 5, 3, 16), order="F")
    q[:, :, 2] = 1.0
    mod.set("topography", np.ones((5, 5, 1, 16), order="F"))
    mod.set("solution", q)
    mod.rk3(20, 1e-3)
    s = mod.get("solution", (5, 5, 3, 16))
    assert np.abs(s[:, :, 0]).max() <= 1000 * np.finfo(float).eps
    assert np.abs(s[:, :, 1]).max() <= 1000 * np.finfo(float).eps


def test_cig_discrete_conservation_periodic():
    m = O.Mesh(4, 4, periodic=(True, True), amp=0.05)
    mod = O.Model(O.CIG, 4, m)
    g = O.Geometry(4, m)
    q = _cig_state(g.x, lambda X, Y: 1 + 0.2 * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y), 0.5, 0.3, 1.0)
    mod.set("solution", q)
    d = mod.tendency()
    w = mod_weights = O.Lagrange(4).qWeights
    wJ = g.J[:, :, 0, :] * w[:, None, None] * w[None, :, None]
    tot = np.einsum("ijve,ije->v", d, wJ)
    assert np.abs(tot).max() < 1e-12, tot
    del mod_weights


def test_lsw_energy_nonincreasing_reflecting_box():
    m = O.Mesh(4, 4, bcid=O.BC_NONORMALFLOW)
    mod = O.Model(O.LSW, 5, m)
    x = O.Geometry(5, m).x
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    q = np.zeros((6, 6, 3, 16), order="F")
    q[:, :, 2] = 0.01 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
    mod.set("H", np.ones((6, 6, 1, 16), order="F"))
    mod.set("solution", q)
    e0 = mod.entropy()
    mod.rk3(50, 2e-3)
    e1 = mod.entropy()
    assert np.isfinite(e1) and e1 <= e0 * (1 + 1e-12)


def test_oracle_regression_vectors():
    from tests.golden import make_golden as mg  # noqa: F401  (fixture generator lives beside the data)
    ref = np.load(os.path.join(GOLD, "oracle_regression.npz"))
    got = mg.regression()
    for k in ref.files:
        np.testing.assert_allclose(got[k], ref[k], rtol=0, atol=0, err_msg=k)


def test_oracle_thread_count_does_not_change_results():
    m = O.Mesh(5, 5, periodic=(True, True), amp=0.05)
    q = _cig_state(O.Geometry(4, m).x, lambda X, Y: 1 + 0.1 * np.sin(2 * np.pi * X), 0.5, 0.3, 1.0)
    outs = []
    for nt in (1, 4):
        O.set_threads(nt)
        mod = O.Model(O.CIG, 4, m)
        mod.set("solution", q)
        mod.rk3(2, 1e-3)
        outs.append(mod.get("solution"))
    np.testing.assert_array_equal(outs[0], outs[1])


def test_gauss_n1_keeps_the_reference_fill_from_the_output_arrays():
    """The reference's LegendreGauss at N = 1 (src/SELF_Quadrature.f90:217-222)
    sets node 1 and weight 1 from its output arguments nodes(0) and
    weights(0), not from the node it has just computed; with the zeroed arrays
    Lagrange%Init passes, the second node is -0 with weight 0.  Library and
    oracle keep that behaviour (so N = 1 Gauss models are not usable, as in
    the reference); every other degree is the Gauss rule."""
    import self_b200 as S
    L = S.Lagrange(1)
    assert L.controlPoints[0] == -np.sqrt(1.0 / 3.0) and L.controlPoints[1] == 0.0
    assert L.qWeights[0] == 1.0 and L.qWeights[1] == 0.0
    x, w = O.quadrature(1, O.GAUSS)
    np.testing.assert_array_equal(x, L.controlPoints)
    np.testing.assert_array_equal(w, L.qWeights)


def _block2d_mesh(bc):
    """The reference's Block2D mesh (etc/mesh/Block2D, pinned above) with every
    physical side set to `bc` (Mesh2D%ResetBoundaryConditionType)."""
    ref = json.load(open(os.path.join(GOLD, "reference_meshes.json")))["Block2D"]
    nx, ny, x0, x1, y0, y1 = ref["structured"]
    return O.Mesh(nx, ny, x0, x1, y0, y1, bcid=bc)


@pytest.mark.parametrize("bc", [O.BC_PRESCRIBED, O.BC_NONORMALFLOW])
def test_cig_static_fluid_stays_static(bc):
    # test/CompressibleIdealGas2D_StaticFluid.f90 (prescribed sides from the
    # initial state) and CompressibleIdealGas2D_StaticFluid_NoNormalFlow.f90
    # (walls): a fluid at rest on Block2D at the CLI defaults (N = 7, Gauss,
    # dt = 5e-4, end time 0.01 = 20 steps).  The reference asserts a finite
    # entropy; in exact arithmetic the state does not move, so the tendency is
    # rounding noise and the entropy (CalculateEntropy, zero for a fluid at
    # rest) is unchanged.
    N, P = 7, 8
    m = _block2d_mesh(bc)
    mod = O.Model(O.CIG, N, m)
    q = np.zeros((P, P, 4, m.nEl), order="F")
    q[:, :, 2] = 1.0
    q[:, :, 3] = 1.0 / 0.4  # p = 1 with gamma = 1.4
    mod.set("solution", q)
    if bc == O.BC_PRESCRIBED:
        mod.set("prescribed")
    e0 = mod.entropy()
    assert np.abs(mod.tendency()).max() < 1e-10
    mod.rk3(20, 5e-4)
    s = mod.get("solution", (P, P, 4, m.nEl))
    assert np.abs(s - q).max() < 1e-12
    e1 = mod.entropy()
    assert np.isfinite(e1) and abs(e1 - e0) <= 1e-12


def test_cig_constant_velocity_prescribed_sides():
    # test/CompressibleIdealGas2D_ConstantVelocity.f90: a uniform flow on
    # Block2D with the prescribed exterior state equal to it; the free stream is
    # an exact steady solution, so the tendency is rounding noise.
    N, P = 7, 8
    m = _block2d_mesh(O.BC_PRESCRIBED)
    mod = O.Model(O.CIG, N, m)
    u, v = 0.5, 0.25
    q = np.zeros((P, P, 4, m.nEl), order="F")
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = u, v, 1.0
    q[:, :, 3] = 1.0 / 0.4 + 0.5 * (u * u + v * v)
    mod.set("solution", q)
    mod.set("prescribed")
    assert np.abs(mod.tendency()).max() < 1e-10
    mod.rk3(20, 5e-4)
    assert np.abs(mod.get("solution", (P, P, 4, m.nEl)) - q).max() < 1e-11


@pytest.mark.parametrize("kind", ["BR", "SF"])
def test_gradient_known_answer_geophysical_mesh(kind):
    # test/GradientBR_Test.f90 and test/GradientSF_Test.f90: on the reference's
    # GeophysicalBlock2DMedium mesh (10 x 10 elements on [-5e5, 5e5]^2, pinned
    # above) at N = 7, s = sin(2 pi x / 1e6) sin(2 pi y / 1e6) with a zero
    # exterior state on the physical sides (extBoundary = 0), against the exact
    # gradient (the reference writes both fields out; s vanishes on the
    # boundary, so the exterior state is consistent with it).
    ref = json.load(open(os.path.join(GOLD, "reference_meshes.json")))["GeophysicalBlock2DMedium"]
    nx, ny, x0, x1, y0, y1 = ref["structured"]
    m = O.Mesh(nx, ny, x0, x1, y0, y1, bcid=O.BC_PRESCRIBED)
    N, P = 7, 8
    L = O.Lagrange(N, O.GAUSS, N, O.UNIFORM)
    g = O.Geometry(N, m)
    X, Y = g.x[0, :, :, 0, :], g.x[1, :, :, 0, :]
    k = 2 * np.pi / 1e6
    f = np.asfortranarray((np.sin(k * X) * np.sin(k * Y)).reshape(P, P, 1, m.nEl, order="F"))
    if kind == "BR":
        fb = O.scalar_boundary_interp(L, f)
        ext = O.side_exchange_scalar(fb, m.sideInfo)  # physical sides keep 0
        grad = O.gradient_br(L, f, O.bassi_rebay_sides(fb, ext), g.dsdx, g.J, g.nHat, g.nScale)
    else:
        grad = O.gradient_sf(L, f, g.dsdx, g.J)
    exact = np.stack([k * np.cos(k * X) * np.sin(k * Y), k * np.sin(k * X) * np.cos(k * Y)])
    err = np.abs(grad[:, :, :, 0, :] - exact).max() / np.abs(exact).max()
    assert err < 1e-8, err  # 2.2e-9 (BR), 2.4e-9 (SF): spectral accuracy at N = 7


@pytest.mark.parametrize("wave", ["planetary", "topographic"])
def test_lsw_rossby_wave_scenarios(wave):
    # test/LinearShallowWater2D_PlanetaryRossbyWave.f90 (f = 1e-4 + 2e-11 y,
    # H = 1000) and LinearShallowWater2D_TopographicRossbyWave.f90 (f = 1e-4,
    # H = 1000 + 2e-4 y): g = 10, eta = 1e-2 exp(-(x^2 + y^2) / 2e10), radiation
    # sides on GeophysicalBlock2DMedium at N = 7.  The reference stops on a
    # non-finite entropy and warns when it grows; both are asserted here over its
    # own run (CLI defaults: 20 steps of 5e-4 s) and over 200 steps of 2 s
    # (gravity waves at 100 m/s, nodes ~1 km apart), where the upwind flux must
    # not add energy.
    ref = json.load(open(os.path.join(GOLD, "reference_meshes.json")))["GeophysicalBlock2DMedium"]
    nx, ny, x0, x1, y0, y1 = ref["structured"]
    m = O.Mesh(nx, ny, x0, x1, y0, y1, bcid=O.BC_RADIATION)
    N, P = 7, 8
    X, Y = (lambda x: (x[0, :, :, 0, :], x[1, :, :, 0, :]))(O.Geometry(N, m).x)
    f = 1e-4 + (2e-11 * Y if wave == "planetary" else 0 * Y)
    H = 1000.0 + (2e-4 * Y if wave == "topographic" else 0 * Y)
    mod = O.Model(O.LSW, N, m, g=10.0)
    mod.set("H", np.asfortranarray(H.reshape(P, P, 1, m.nEl, order="F")))
    mod.set("fCori", np.asfortranarray(f.reshape(P, P, 1, m.nEl, order="F")))
    q = np.zeros((P, P, 3, m.nEl), order="F")
    q[:, :, 2] = 1e-2 * np.exp(-(X ** 2 + Y ** 2) / 2e10)
    mod.set("solution", q)
    e0 = mod.entropy()
    mod.rk3(20, 5e-4)
    e1 = mod.entropy()
    assert np.isfinite(e1) and e1 <= e0 * (1 + 1e-12)
    mod.rk3(200, 2.0)
    e2 = mod.entropy()
    assert np.isfinite(e2) and e2 <= e1 * (1 + 1e-12)
    assert e2 < e1  # the upwind flux dissipates (relative 6e-10 over these 400 s)
