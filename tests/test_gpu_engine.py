"""Parity of the fused CUDA engine (libselfgpu) with the FP64 CPU oracle.

Tolerance: 1e-12 relative (max abs difference over max abs reference value,
per field) for the tendency and after RK3 steps -- the bar both FP64 forms
are held to: the production form (FP64, multiply-add contraction and
reciprocal products) and the reference-rounding form (FP64_REF), which in
addition equals the oracle bit for bit.  Every case runs the reference's call
order: mesh -> geometry -> model fields -> SetSolution -> CalculateTendency /
ForwardStep.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu
TOL = 1e-12
FORMS = [0, 2]  # self_b200.FP64 (production), self_b200.FP64_REF (reference roundings)


def build_oracle(model, mesh_kind, N, seed=0, fast=False):
    """The oracle half of build_pair; fast=True builds it from the oracle's
    multiply-add-contracted build (a second valid FP64 rounding of the same
    reference loops)."""
    kw = C.mesh_kwargs(mesh_kind)
    om = C.oracle_mesh(kw)
    mod_o = O.Model(C.MODELS[model], N, om, fast=fast)
    x = O.Geometry(N, om).x
    aux = C.aux_fields(model, x, seed)
    if model == "LSW":
        mod_o.set("H", aux["H"])
        mod_o.set("fCori", aux["fCori"])
    elif model == "SW":
        mod_o.set("topography", aux["topography"])
    else:
        mod_o.set("gravityPotential", aux["gravityPotential"])
        mod_o.set("drag", aux["drag"])
    mod_o.set("solution", C.initial_state(model, x, seed))
    if model == "CIG" and kw.get("bcid") in (O.BC_PRESCRIBED, O.BC_RADIATION):
        mod_o.set("prescribed")
    return mod_o


def check_tendency(got, ref, form, model, mesh_kind, N, seed):
    """Tendency parity.  Reference-rounding form: 1e-12 relative per field
    (max |difference| / max |oracle value|; it is bit-exact in practice).
    Production form: per field, within 1e-12 relative or within 8x the
    oracle's own sensitivity to rounding order on the same inputs (its
    contracted build against its plain build), whichever is larger.  Where a
    field's tendency is a small difference of large weak-form terms (the
    ShallowWater thickness on periodic meshes, the density at 128 x 128), any
    change of rounding order moves it by more than 1e-12 of its own size, the
    reference's too."""
    import self_b200 as S
    if form == S.FP64_REF:
        for v in range(ref.shape[2]):
            assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))
        return
    alt = build_oracle(model, mesh_kind, N, seed, fast=True).tendency()
    for v in range(ref.shape[2]):
        scale = np.abs(ref[:, :, v]).max()
        sens = np.abs(alt[:, :, v] - ref[:, :, v]).max()
        diff = np.abs(got[:, :, v] - ref[:, :, v]).max()
        assert diff <= max(TOL * scale, 8.0 * sens), (v, diff / scale, sens / scale)


def build_pair(model, mesh_kind, N, seed=0, form=0):
    import self_b200 as S
    kw = C.mesh_kwargs(mesh_kind)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    mod_o = O.Model(C.MODELS[model], N, om)
    geo_o = O.Geometry(N, om)
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    geo = S.SEMQuad(interp, pm)
    cls = {"LSW": S.LinearShallowWater, "SW": S.ShallowWater, "CIG": S.CompressibleIdealGas2D}[model]
    mod = cls(pm, geo, form=form)
    aux = C.aux_fields(model, geo_o.x, seed)
    if model == "LSW":
        mod_o.set("H", aux["H"])
        mod_o.set("fCori", aux["fCori"])
        mod.SetBathymetry(aux["H"])
        mod.SetCoriolis(aux["fCori"])
    elif model == "SW":
        mod_o.set("topography", aux["topography"])
        mod.SetTopography(aux["topography"])
    else:
        mod_o.set("gravityPotential", aux["gravityPotential"])
        mod_o.set("drag", aux["drag"])
        mod.SetGravity(aux["gravityPotential"])
        mod.SetDrag(aux["drag"])
    q0 = C.initial_state(model, geo_o.x, seed)
    mod_o.set("solution", q0)
    mod.SetSolution(q0)
    if model == "CIG" and kw.get("bcid") in (O.BC_PRESCRIBED, O.BC_RADIATION):
        mod_o.set("prescribed")
        mod.SetPrescribedSolution()
    return mod_o, mod, geo_o, geo


@pytest.mark.parametrize("N", [2, 3, 5, 7])
def test_device_geometry_matches_oracle(N):
    import self_b200 as S
    kw = C.mesh_kwargs("flipped")
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    g_o = O.Geometry(N, om)
    g = S.SEMQuad(S.Lagrange(N), pm)
    for name in ("x", "dxds", "dsdx", "J", "nHat", "nScale"):
        got = S.to_host(getattr(g, name)).reshape(getattr(g_o, name).shape, order="F")
        assert C.rel_err(got, getattr(g_o, name)) < 1e-14, name
    assert abs(g.CovariantArcMin() - g_o.arcmin) < 1e-13 * g_o.arcmin


CASES = [(m, k) for m in ("LSW", "SW", "CIG") for k in ("periodic", "walls", "flipped", "radiation")] + \
        [("CIG", "prescribed")]


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("N", [2, 3, 4, 7])  # odd and even P; P*P < 4P at N = 2
@pytest.mark.parametrize("model,mesh_kind", CASES)
def test_tendency_matches_oracle(model, mesh_kind, N, form):
    import self_b200 as S
    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, form=form)
    ref = mod_o.tendency()
    got = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    check_tendency(got, ref, form, model, mesh_kind, N, 0)
    # a second call with the same solution gives the same tendency (trace cache reuse)
    got2 = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    if model != "SW":  # SW's velocity traces lag one call behind the solution traces by design
        np.testing.assert_array_equal(got2, got)


@pytest.mark.parametrize("model,mesh_kind", [("LSW", "walls"), ("SW", "flipped"), ("CIG", "periodic"),
                                             ("CIG", "prescribed")])
def test_fp64_tendency_and_steps_are_bit_exact(model, mesh_kind):
    """The reference-rounding FP64 form evaluates every expression in the
    reference's order with IEEE roundings and no multiply-add contraction, on
    geometry built the same way: tendency and RK3 states equal the oracle's
    bit for bit."""
    import self_b200 as S
    N = 7
    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, seed=2, form=S.FP64_REF)
    ref = mod_o.tendency()
    got = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    np.testing.assert_array_equal(got, ref)
    mod_o2, mod2, _, _ = build_pair(model, mesh_kind, N, seed=2, form=S.FP64_REF)
    mod_o2.rk3(4, 1e-3)
    mod2.ForwardStep(4, 1e-3)
    ref = mod_o2.get("solution", ref.shape)
    np.testing.assert_array_equal(S.to_host(mod2.solution).reshape(ref.shape, order="F"), ref)


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("N", [2, 5])
@pytest.mark.parametrize("model,mesh_kind", CASES)
def test_rk3_steps_match_oracle(model, mesh_kind, N, form):
    import self_b200 as S
    n, dt = 12, 1e-3
    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, seed=3, form=form)
    mod_o.rk3(n, dt)
    mod.ForwardStep(n, dt)
    ref = mod_o.get("solution", (N + 1, N + 1, mod.nVar, mod.nElem))
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    for v in range(ref.shape[2]):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("model", ["LSW", "SW", "CIG"])
def test_100_rk3_steps_match_oracle(model, form):
    import self_b200 as S
    N, dt = 7, 5e-4
    mesh_kind = "periodic" if model == "CIG" else "walls"
    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, seed=7, form=form)
    mod_o.rk3(100, dt)
    mod.ForwardStep(40, dt)  # split calls: graph replay across calls keeps the state
    mod.ForwardStep(60, dt)
    ref = mod_o.get("solution", (N + 1, N + 1, mod.nVar, mod.nElem))
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    for v in range(ref.shape[2]):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))
    mod.CheckFinite()


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("N", [4, 7])  # the per-element kernel (odd P) and the persistent kernel
@pytest.mark.parametrize("model", ["LSW", "SW", "CIG"])
@pytest.mark.parametrize("mesh_kind", ["single", "column", "row", "pair", "ring", "torus"])
def test_edge_meshes(model, mesh_kind, N, form):
    """Meshes at the edges of the layout: one element (all four sides
    physical), one column and one row of elements (fewer elements than SMs,
    so fewer CTAs than the persistent grid), the smallest periodic mesh,
    where each element is the neighbour of another on two sides and rotated
    elements meet with flipped sides, and periodic directions one element
    wide, where a side's neighbour is its own element.  Tendency and RK3
    steps equal the oracle's bit for bit in the reference-rounding form and
    within 1e-12 in the production form."""
    import self_b200 as S

    def same(got, ref):
        if form == S.FP64_REF:
            np.testing.assert_array_equal(got, ref)
        else:
            for v in range(ref.shape[2]):
                assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))

    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, seed=5, form=form)
    ref = mod_o.tendency()
    got = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    assert np.isfinite(ref).all()
    if form == S.FP64_REF:
        same(got, ref)
    else:
        check_tendency(got, ref, form, model, mesh_kind, N, 5)
    mod_o2, mod2, _, _ = build_pair(model, mesh_kind, N, seed=5, form=form)
    mod_o2.rk3(5, 1e-3)
    mod2.ForwardStep(5, 1e-3)
    ref = mod_o2.get("solution", ref.shape)
    same(S.to_host(mod2.solution).reshape(ref.shape, order="F"), ref)


@pytest.mark.parametrize("form", FORMS)
def test_c2_full_size_tendency_and_steps(form):
    """The CompressibleIdealGas2D benchmark workload at full size: periodic
    128x128, perturbed nodes (0.02 h), N = 7: tendency and 2 RK3 steps against
    the oracle, plus free-stream preservation and discrete conservation."""
    import os

    import self_b200 as S
    O.set_threads(os.cpu_count() or 1)
    N, nx = 7, 128
    kw = dict(nx=nx, ny=nx, periodic=(True, True), amp=0.02)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    geo_o = O.Geometry(N, om)
    mod_o = O.Model(O.CIG, N, om)
    geo = S.SEMQuad(S.Lagrange(N), pm)
    mod = S.CompressibleIdealGas2D(pm, geo, form=form)
    X, Y = geo_o.x[0, :, :, 0, :], geo_o.x[1, :, :, 0, :]
    q = np.zeros((8, 8, 4, nx * nx), order="F")
    rho = 1 + 0.1 * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y)
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * 0.5, rho * 0.3, rho
    q[:, :, 3] = 1.0 / 0.4 + 0.5 * rho * 0.34
    mod_o.set("solution", q)
    mod.SetSolution(q)
    ref = mod_o.tendency()
    got = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    if form == S.FP64_REF:
        for v in range(4):
            assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL
    else:  # the bound of check_tendency: 1e-12 or 8x the oracle's own rounding sensitivity
        alt_o = O.Model(O.CIG, N, om, fast=True)
        alt_o.set("solution", q)
        alt = alt_o.tendency()
        for v in range(4):
            scale = np.abs(ref[:, :, v]).max()
            sens = np.abs(alt[:, :, v] - ref[:, :, v]).max()
            diff = np.abs(got[:, :, v] - ref[:, :, v]).max()
            assert diff <= max(TOL * scale, 8.0 * sens), (v, diff / scale, sens / scale)
    # discrete conservation: sum of J w_i w_j dSdt vanishes on a periodic mesh
    w = S.Lagrange(N).qWeights
    wJ = geo_o.J[:, :, 0, :] * w[:, None, None] * w[None, :, None]
    tot = np.einsum("ijve,ije->v", got, wJ)
    assert np.abs(tot).max() < 1e-10 * np.abs(got).max()
    dt = 1e-4
    mod_o.rk3(2, dt)
    mod.ForwardStep(2, dt)
    ref = mod_o.get("solution", q.shape)
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    for v in range(4):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL
    # free stream on the same perturbed mesh
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = 0.5, 0.3, 1.0
    q[:, :, 3] = 1.0 / 0.4 + 0.5 * 0.34
    mod.SetSolution(q)
    d = mod.CalculateTendency()
    # round-off of the metric identities at h = 1/128 (the oracle's residual is the same, bit for bit,
    # in the reference-rounding form)
    assert float(d.abs().max()) < 1e-6
    torch.cuda.synchronize()


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("model", ["LSW", "SW", "CIG"])
@pytest.mark.parametrize("N", [3, 7])
def test_persistent_kernel_matches_per_element_kernel(model, N, form):
    """The persistent bulk-copy kernel and the per-element-group kernel compute
    the same values: bit-identical states after RK3 steps in the
    reference-rounding form, within 1e-12 in the production form (the two
    kernels group their multiply-adds differently)."""
    import self_b200 as S
    n, dt = 6, 1e-3
    mesh_kind = "periodic" if model == "CIG" else "flipped"
    outs = []
    for persistent in (1, 0):
        _, mod, _, _ = build_pair(model, mesh_kind, N, seed=5, form=form)
        S.check(S.lib().selfgpu_model2d_set_launch(mod._h, persistent, 0))
        mod.ForwardStep(n, dt)
        mod.Sync()
        if persistent:
            assert S.lib().selfgpu_model2d_persistent_launch_count(mod._h) == 3 * n
        outs.append(S.to_host(mod.solution).copy())
    if form == S.FP64_REF:
        np.testing.assert_array_equal(outs[0], outs[1])
    else:
        for v in range(outs[1].shape[2]):
            assert C.rel_err(outs[0][:, :, v], outs[1][:, :, v]) < TOL


@pytest.mark.parametrize("model,N", [("CIG", 7), ("SW", 5), ("LSW", 7)])
def test_rk3_graph_steps_match_separate_stage_launches_bitwise(model, N):
    """On a mesh with several elements per CTA, ForwardStep (graph-replayed
    steps, each stage launched as a programmatic dependent of the previous
    one) and the same stages issued one by one through selfgpu_model2d_stage
    (the multi-rank entry point) give bit-identical states over two calls."""
    import self_b200 as S
    L = S.lib()
    n, dt = 4, 2e-4
    outs = []
    for graphed in (True, False):
        mesh = S.Mesh2D(24, 20, periodic=(True, True), perturbation=0.05)
        geo = S.SEMQuad(S.Lagrange(N, S.GAUSS, N, S.UNIFORM), mesh)
        cls = {"LSW": S.LinearShallowWater, "SW": S.ShallowWater, "CIG": S.CompressibleIdealGas2D}[model]
        mod = cls(mesh, geo)
        x = S.to_host(geo.x)
        aux = C.aux_fields(model, x, 9)
        if model == "LSW":
            mod.SetBathymetry(aux["H"])
            mod.SetCoriolis(aux["fCori"])
        elif model == "SW":
            mod.SetTopography(aux["topography"])
        else:
            mod.SetGravity(aux["gravityPotential"])
            mod.SetDrag(aux["drag"])
        mod.SetSolution(C.initial_state(model, x, 9))
        if graphed:
            mod.ForwardStep(n, dt)
            mod.ForwardStep(n, dt)
        else:
            S.check(L.selfgpu_model2d_prologue(mod._h))
            for _ in range(2 * n):
                for st in range(3):
                    S.check(L.selfgpu_model2d_stage(mod._h, dt, st))
        mod.Sync()
        outs.append(S.to_host(mod.solution).copy())
    assert np.isfinite(outs[0]).all()
    np.testing.assert_array_equal(outs[0], outs[1])


def test_bounded_wait_timeout_is_reported_and_context_survives():
    """A stalled copy (registered, never issued) makes the consumers' bounded
    wait run out: the kernel returns, sync reports SELFGPU_ERR_TIMEOUT (6), and
    the engine runs normally afterwards."""
    import self_b200 as S
    _, mod, _, _ = build_pair("CIG", "periodic", 7)
    L = S.lib()
    assert L.selfgpu_model2d_set_wait_limit(mod._h, 100_000_000) == 0  # ~50 ms
    assert L.selfgpu_model2d_inject_stall(mod._h, 1) == 0
    mod.ForwardStep(1, 1e-3)
    with pytest.raises(S.SelfGpuError) as ei:
        mod.Sync()
    assert ei.value.code == 6
    L.selfgpu_model2d_inject_stall(mod._h, 0)
    mod.SetSolution(torch.ones_like(mod.solution) + 1.0)
    mod.ForwardStep(2, 1e-3)
    mod.Sync()
    mod.CheckFinite()


@pytest.mark.parametrize("model,mesh_kind,N", [("CIG", "periodic", 7), ("SW", "walls", 5), ("LSW", "walls", 5)])
def test_fp32_bulk_form_error_vs_fp64_oracle(model, mesh_kind, N, capsys):
    """FP32-bulk form (float fluxes, traces and divergence; FP64 metrics,
    sources, 1/J and RK accumulation): relative L2 error against the FP64
    oracle after 40 RK3 steps on smooth states."""
    import self_b200 as S
    kw = C.mesh_kwargs(mesh_kind)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    mod_o = O.Model(C.MODELS[model], N, om)
    geo_o = O.Geometry(N, om)
    geo = S.SEMQuad(S.Lagrange(N), pm)
    cls = {"LSW": S.LinearShallowWater, "SW": S.ShallowWater, "CIG": S.CompressibleIdealGas2D}[model]
    mod = cls(pm, geo, form=S.FP32_BULK)
    aux = C.aux_fields(model, geo_o.x, 0)
    if model == "LSW":
        mod_o.set("H", aux["H"])
        mod.SetBathymetry(aux["H"])
    elif model == "SW":
        mod_o.set("topography", aux["topography"])
        mod.SetTopography(aux["topography"])
    q0 = C.initial_state(model, geo_o.x, 0)
    mod_o.set("solution", q0)
    mod.SetSolution(q0)
    mod_o.rk3(40, 1e-3)
    mod.ForwardStep(40, 1e-3)
    ref = mod_o.get("solution", q0.shape)
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    with capsys.disabled():
        print(f"\nFP32-bulk {model} N={N}: relative L2 error after 40 steps = {err:.3e}")
    assert err < 1e-6  # the bar for the mixed-precision forms on smooth cases


def test_engine_rejects_malformed_side_info():
    import self_b200 as S
    pm = C.product_mesh(C.mesh_kwargs("periodic"))
    pm.sideInfo[2, 1, 3] = 999
    geo = S.SEMQuad(S.Lagrange(3), C.product_mesh(C.mesh_kwargs("periodic")))
    with pytest.raises(S.SelfGpuError) as ei:
        S.CompressibleIdealGas2D(pm, geo)
    assert ei.value.code == 2


def test_check_finite_flags_injected_nan():
    import self_b200 as S
    mod_o, mod, _, _ = build_pair("CIG", "periodic", 3)
    mod.CheckFinite()
    mod.solution[0, 2, 1, 1] = float("nan")  # injected on the host side of the API
    with pytest.raises(S.SelfGpuError) as ei:
        mod.CheckFinite()
    assert ei.value.code == 5


@pytest.mark.parametrize("form", FORMS)
def test_checkpoint_pickup_continues(tmp_path, form):
    """Write_Model2D after some steps, Read_Model2D into a fresh model: the
    continued run equals the uninterrupted one (the first RK3 stage multiplies
    the RK register by a_1 = 0, so the solution is the whole state) bit for
    bit in the reference-rounding form; in the production form within 1e-12
    (a pickup rebuilds the face-trace cache with the per-element kernel, whose
    multiply-adds the compiler may group differently from the persistent
    kernel's), and the file carries the reference's dataset paths and shapes."""
    import self_b200 as S
    from self_b200.checkpoint import Checkpoint
    N, dt = 5, 1e-3
    _, a, _, _ = build_pair("CIG", "periodic", N, seed=9, form=form)
    _, b, _, _ = build_pair("CIG", "periodic", N, seed=9, form=form)
    a.ForwardStep(6, dt)
    name = a.Write(str(tmp_path / "pick.ckpt"))
    with Checkpoint(name) as c:
        P, nEl = N + 1, a.nElem
        assert c.attr("N") == N
        assert c.info("/state/interior/solution")[1] == [P, P, 4, nEl]
        assert c.info("/state/boundary/solution")[1] == [P, 4, 4, nEl]
        assert c.info("/mesh/interior/x")[1] == [2, P, P, 1, nEl]
        assert c.info("/mesh/boundary/x")[1] == [2, P, 1, 4, nEl]
        assert c.info("/quadrature/dgmatrix")[1] == [P, P]
        np.testing.assert_array_equal(c.get("/state/interior/solution"), S.to_host(a.solution))
    a.ForwardStep(5, dt)
    b.Read(name)
    assert b.t == pytest.approx(6 * dt)
    b.ForwardStep(5, dt)
    if form == S.FP64_REF:
        np.testing.assert_array_equal(S.to_host(b.solution), S.to_host(a.solution))
    else:
        assert C.rel_err(S.to_host(b.solution), S.to_host(a.solution)) < TOL
    _, wrong, _, _ = build_pair("CIG", "periodic", 3, seed=9)
    with pytest.raises(S.SelfGpuError):
        wrong.Read(name)


@pytest.mark.parametrize("form", FORMS)
def test_c1_gravity_wave_release_1000_steps(form):
    """The LinearShallowWater gravity-wave release exactly as configured for
    the reference's CPU-runnable case: 10x10 walls, N = 7 Legendre-Gauss,
    g = H = 1, f = 0, eta0 = 0.01 exp(-r^2 / 0.1^2), u = v = 0, Rusanov flux,
    RK3 with dt = 1e-4 for 1000 steps: the state equals the oracle's bit for
    bit in the reference-rounding form and within 1e-12 in the production
    form."""
    import self_b200 as S
    N, dt, steps = 7, 1e-4, 1000
    kw = dict(nx=10, ny=10, bcid=O.BC_NONORMALFLOW, amp=0.0)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    mod_o = O.Model(C.MODELS["LSW"], N, om)
    geo_o = O.Geometry(N, om)
    geo = S.SEMQuad(S.Lagrange(N, S.GAUSS, N, S.UNIFORM), pm)
    mod = S.LinearShallowWater(pm, geo, form=form)
    X, Y = geo_o.x[0, :, :, 0, :], geo_o.x[1, :, :, 0, :]
    P = N + 1
    q0 = np.zeros((P, P, 3, X.shape[2]), order="F")
    q0[:, :, 2] = 0.01 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
    H = np.ones((P, P, 1, X.shape[2]), order="F")
    f = np.zeros((P, P, 1, X.shape[2]), order="F")
    mod_o.set("H", H)
    mod_o.set("fCori", f)
    mod.SetBathymetry(H)
    mod.SetCoriolis(f)
    mod_o.set("solution", q0)
    mod.SetSolution(q0)
    mod_o.rk3(steps, dt)
    mod.ForwardStep(steps, dt)
    mod.Sync()
    ref = mod_o.get("solution", q0.shape)
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    if form == S.FP64_REF:
        np.testing.assert_array_equal(got, ref)
    else:
        for v in range(3):
            assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))
    assert np.isfinite(got).all() and np.abs(got[:, :, 2]).max() > 1e-4


@pytest.mark.parametrize("model,mesh_kind", [("LSW", "walls"), ("SW", "flipped"), ("CIG", "periodic"),
                                             ("CIG", "prescribed")])
def test_entropy_matches_oracle(model, mesh_kind):
    """CalculateEntropy reduced on the device against the oracle's
    restatement of the reference loops, before and after RK3 steps (the
    oracle's CompressibleIdealGas2D entropy reads the primitive field of its
    last tendency, so a tendency call refreshes it first)."""
    N, n, dt = 5, 6, 1e-3
    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, seed=4)
    for k in range(2):
        if k:
            mod_o.rk3(n, dt)
            mod.ForwardStep(n, dt)
        mod_o.tendency()
        e_o = mod_o.entropy()
        e = mod.CalculateEntropy()
        assert e_o != 0.0 and abs(e - e_o) <= 1e-12 * abs(e_o), (k, e, e_o)


@pytest.mark.parametrize("form", FORMS)
def test_c1_one_launch_1000_steps(form):
    """The gravity-wave release (LSW 10x10 walls, N = 7, dt = 1e-4) with all
    3000 RK stages in one cooperative launch: equal to the oracle bit for bit
    in the reference-rounding form, within 1e-12 in the production form."""
    import self_b200 as S
    N, dt, steps = 7, 1e-4, 1000
    kw = dict(nx=10, ny=10, bcid=O.BC_NONORMALFLOW, amp=0.0)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    mod_o = O.Model(C.MODELS["LSW"], N, om)
    geo_o = O.Geometry(N, om)
    geo = S.SEMQuad(S.Lagrange(N, S.GAUSS, N, S.UNIFORM), pm)
    mod = S.LinearShallowWater(pm, geo, form=form)
    S.check(S.lib().selfgpu_model2d_set_multistep(mod._h, 1))
    X, Y = geo_o.x[0, :, :, 0, :], geo_o.x[1, :, :, 0, :]
    P = N + 1
    q0 = np.zeros((P, P, 3, X.shape[2]), order="F")
    q0[:, :, 2] = 0.01 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
    H = np.ones((P, P, 1, X.shape[2]), order="F")
    f = np.zeros((P, P, 1, X.shape[2]), order="F")
    for m_ in (mod_o,):
        m_.set("H", H)
        m_.set("fCori", f)
        m_.set("solution", q0)
    mod.SetBathymetry(H)
    mod.SetCoriolis(f)
    mod.SetSolution(q0)
    l0 = mod.LaunchCount()
    mod.ForwardStep(steps, dt)
    mod.Sync()
    assert mod.LaunchCount() - l0 <= 2  # the trace prologue and the one multi-stage launch
    mod_o.rk3(steps, dt)
    ref = mod_o.get("solution", q0.shape)
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    assert np.isfinite(got).all()
    if form == S.FP64_REF:
        np.testing.assert_array_equal(got, ref)
    else:
        for v in range(3):
            assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))


@pytest.mark.parametrize("model,mesh_kind,N", [("SW", "flipped", 5), ("CIG", "prescribed", 4), ("LSW", "periodic", 3)])
def test_one_launch_steps_match_oracle(model, mesh_kind, N):
    """One cooperative launch for several RK3 steps, over two calls (odd step
    counts, so the trace-cache parity flips between them), for every model:
    the reference-rounding form equals the oracle bit for bit."""
    import self_b200 as S
    mod_o, mod, _, _ = build_pair(model, mesh_kind, N, seed=8, form=S.FP64_REF)
    S.check(S.lib().selfgpu_model2d_set_multistep(mod._h, 1))
    mod.ForwardStep(3, 1e-3)
    mod.ForwardStep(4, 1e-3)
    mod.Sync()
    mod_o.rk3(7, 1e-3)
    ref = mod_o.get("solution", (N + 1, N + 1, mod.nVar, mod.nElem))
    np.testing.assert_array_equal(S.to_host(mod.solution).reshape(ref.shape, order="F"), ref)


def test_one_launch_falls_back_on_a_mesh_larger_than_one_wave():
    """A mesh whose element groups exceed one wave of resident CTAs runs the
    graph-replayed steps instead, with the same result."""
    import self_b200 as S
    outs = []
    for ms in (1, 0):
        mesh = S.Mesh2D(96, 96, periodic=(True, True))
        geo = S.SEMQuad(S.Lagrange(7), mesh)
        mod = S.CompressibleIdealGas2D(mesh, geo, form=S.FP64_REF)
        S.check(S.lib().selfgpu_model2d_set_multistep(mod._h, ms))
        X, Y = geo.x[..., 0], geo.x[..., 1]
        rho = 1.0 + 0.1 * torch.sin(2 * np.pi * X) * torch.sin(2 * np.pi * Y)
        q = torch.stack([rho * 0.5, rho * 0.3, rho, 2.5 + 0.17 * rho], dim=1)[:, :, 0].contiguous()
        mod.SetSolution(q)
        mod.ForwardStep(3, 1e-4)
        mod.Sync()
        outs.append(mod.solution.clone())
    assert torch.equal(outs[0], outs[1])


def _multistage_pair(model, walls, form, nx=80, N=7):
    """Two identical handles on an nx x nx mesh (N = 7: one element per
    group, at least three per group and stage from 4 440 elements, 5 328 for
    the kernels that run twelve groups, 6 216 for fourteen), the first with
    multi-stage launches on."""
    import self_b200 as S
    L = S.lib()
    kw = dict(bcid=S.BC_NONORMALFLOW) if walls else dict(periodic=(True, True), perturbation=0.02)
    out = []
    for multi in (1, 0):
        interp = S.Lagrange(N)
        mesh = S.Mesh2D(nx, nx, **kw)
        geo = S.SEMQuad(interp, mesh)
        cls = {"LSW": S.LinearShallowWater, "SW": S.ShallowWater, "CIG": S.CompressibleIdealGas2D}[model]
        m = cls(mesh, geo, form=form)
        X, Y = geo.x[:, 0, :, :, 0], geo.x[:, 0, :, :, 1]
        P = N + 1
        q = torch.zeros((mesh.nElem, 4 if model == "CIG" else 3, P, P), device="cuda", dtype=torch.float64)
        bump = 0.01 * torch.exp(-((X - 0.4) ** 2 + (Y - 0.6) ** 2) / 0.05)
        if model == "CIG":
            rho = 1.0 + 0.1 * torch.sin(2 * np.pi * X) * torch.sin(2 * np.pi * Y)
            q[:, 0], q[:, 1], q[:, 2], q[:, 3] = rho * 0.5, rho * 0.3, rho, 2.5 + 0.17 * rho
        elif model == "SW":
            q[:, 0], q[:, 2] = 0.2 * bump, 1.0 + bump
        else:
            q[:, 2] = bump
        m.SetSolution(q)
        assert L.selfgpu_model2d_set_multistage(m._h, multi) == 0
        assert L.selfgpu_model2d_set_wait_limit(m._h, 400_000_000) == 0  # ~0.2 s
        out.append(m)
    return out


@pytest.mark.parametrize("model,walls", [("CIG", False), ("SW", True), ("LSW", True)])
@pytest.mark.parametrize("form_name", ["FP64", "FP64_REF", "FP32_BULK"])
def test_multistage_launch_equals_stage_launches(model, walls, form_name):
    """All RK stages of an rk3 call in one launch of the persistent kernel
    (elements copied ahead across stage boundaries, a stage-end counter before
    the neighbour reads) give the stage-by-stage launches' state bit for bit,
    over calls of several lengths."""
    import self_b200 as S
    L = S.lib()
    a, b = _multistage_pair(model, walls, getattr(S, form_name))
    dt = 2e-5 if model == "CIG" else 1e-4
    l0 = L.selfgpu_model2d_launch_count(a._h)
    for n in (5, 1, 3):
        a.ForwardStep(n, dt)
        b.ForwardStep(n, dt)
    a.Sync()
    b.Sync()
    assert L.selfgpu_model2d_launch_count(a._h) - l0 == 1 + 3  # the trace prologue, then one launch per call
    assert torch.isfinite(a.solution).all()
    assert torch.equal(a.solution, b.solution) and torch.equal(a.workSol, b.workSol)


def test_multistage_falls_back_where_it_does_not_apply():
    """N = 5 (four-element tiles) and a mesh too small for three elements per
    group: rk3 with multi-stage launches on runs the stage launches."""
    import self_b200 as S
    L = S.lib()
    for model, nx, N in (("SW", 72, 5), ("CIG", 24, 7)):
        a, b = _multistage_pair(model, True, S.FP64, nx=nx, N=N)
        l0 = L.selfgpu_model2d_launch_count(a._h)
        a.ForwardStep(4, 1e-4)
        b.ForwardStep(4, 1e-4)
        a.Sync()
        b.Sync()
        assert L.selfgpu_model2d_launch_count(a._h) - l0 == 1 + 12
        assert torch.equal(a.solution, b.solution)


def test_multistage_stage_end_wait_timeout_is_reported():
    """One group never announces the end of its stages: every other group's
    bounded stage-end wait runs out, sync reports SELFGPU_ERR_TIMEOUT (6), and
    the handle runs normally afterwards."""
    import self_b200 as S
    L = S.lib()
    a, _ = _multistage_pair("CIG", False, S.FP64)
    assert L.selfgpu_model2d_set_wait_limit(a._h, 100_000_000) == 0  # ~50 ms
    assert L.selfgpu_model2d_inject_stall(a._h, 2) == 0
    a.ForwardStep(2, 2e-5)
    with pytest.raises(S.SelfGpuError) as ei:
        a.Sync()
    assert ei.value.code == 6
    assert L.selfgpu_model2d_inject_stall(a._h, 3) != 0
    assert L.selfgpu_model2d_inject_stall(a._h, 0) == 0
    q = torch.empty_like(a.solution)  # a uniform state (positive pressure)
    for v, x in enumerate((0.5, 0.3, 1.0, 2.5)):
        q[:, v] = x
    a.SetSolution(q)
    a.ForwardStep(2, 2e-5)
    a.Sync()
    a.CheckFinite()


def test_multistage_launch_with_element_time_steps():
    """Per-element time steps (the ensembles' elementDt field) in the
    multi-stage launch: bit for bit the stage launches' result."""
    import self_b200 as S
    a, b = _multistage_pair("SW", True, S.FP64)
    nEl = a.solution.shape[0]
    dtE = 1e-4 * (1.0 + 0.5 * torch.rand(nEl, device="cuda", dtype=torch.float64,
                                         generator=torch.Generator(device="cuda").manual_seed(3)))
    for m in (a, b):
        m._set_field("elementDt", dtE)
    a.ForwardStep(4, 0.0)
    b.ForwardStep(4, 0.0)
    a.Sync()
    b.Sync()
    assert torch.isfinite(a.solution).all()
    assert torch.equal(a.solution, b.solution)
