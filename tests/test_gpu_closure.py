"""The shock closure on the GPU against the oracle: features and indicator,
the closure's viscous terms in the tendency and through RK3 steps (1e-12
relative in FP64), the closure MLP's inference against its numpy
restatement, and its training."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _modal_decay_exponent(q, N):
    """s = log10(highest-shell energy / total energy) of the density, per element (numpy)."""
    T = O.modal_matrix(N)
    P = N + 1
    rho = q[:, :, 2, :]
    c = np.einsum("ki,ije,lj->kle", T, rho, T)
    e = c * c
    top = e[N, :, :].sum(axis=0) + e[:N, N, :].sum(axis=0)
    return np.log10(np.maximum(top, 1e-300) / e.sum(axis=(0, 1)))


def _pair(mesh_kind, N, seed=0, c=1.0):
    import self_b200 as S
    kw = C.mesh_kwargs(mesh_kind)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    mod_o = O.Model(O.CIG, N, om)
    geo_o = O.Geometry(N, om)
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    geo = S.SEMQuad(interp, pm)
    mod = S.CompressibleIdealGas2D(pm, geo)
    q0 = C.shock_state(geo_o.x, seed)
    mod_o.set("solution", q0)
    mod.SetSolution(q0)
    if mesh_kind in ("prescribed", "radiation"):
        mod_o.set("prescribed")
        mod.SetPrescribedSolution()
    return mod_o, mod, geo_o, q0


@pytest.mark.parametrize("N", [3, 5, 7])
def test_features_and_indicator_match_oracle(N):
    import self_b200 as S
    from self_b200 import closure as CL
    m = O.Mesh(6, 5, periodic=(True, True), amp=0.03)
    g = O.Geometry(N, m)
    q = C.shock_state(g.x, 2)
    act_o, feat_o = O.closure_features(q, N)
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    act, feat = CL.features(S.to_device(q), interp)
    assert (act_o > 0).any()
    assert np.abs(act.cpu().numpy() - act_o).max() < 1e-6
    if N >= 5:
        assert np.abs(feat.cpu().numpy() - feat_o.T).max() < 1e-5


@pytest.mark.parametrize("N", [3, 5, 7])
@pytest.mark.parametrize("mesh_kind", ["periodic", "walls", "flipped", "prescribed"])
def test_indicator_closure_tendency_matches_oracle(mesh_kind, N):
    import self_b200 as S
    mod_o, mod, _, _ = _pair(mesh_kind, N)
    mod_o.set_closure(1, c=1.0)
    mod.SetClosure(S.CLOSURE_INDICATOR, c=1.0)
    ref = mod_o.tendency()
    got = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    nu_o = mod_o.get("avNu")
    nu, act, _, _ = mod.ClosureState()
    assert nu_o.max() > 0
    assert np.abs(nu.cpu().numpy() - nu_o).max() <= 1e-13 * nu_o.max()
    for v in range(4):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))


@pytest.mark.parametrize("kernel", [1, 0])
def test_indicator_closure_rk3_matches_oracle(kernel):
    import self_b200 as S
    N, n, dt = 5, 10, 2e-4
    mod_o, mod, _, _ = _pair("periodic", N, seed=3)
    S.lib().selfgpu_model2d_set_kernel(mod._h, kernel)
    mod_o.set_closure(1, c=1.0)
    mod.SetClosure(S.CLOSURE_INDICATOR, c=1.0)
    mod_o.rk3(n, dt)
    mod.ForwardStep(4, dt)
    mod.ForwardStep(6, dt)  # graph replay across calls
    ref = mod_o.get("solution", (N + 1, N + 1, 4, mod.nElem))
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    for v in range(4):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, (v, C.rel_err(got[:, :, v], ref[:, :, v]))
    assert mod.LaunchCount() >= 2 * 3 * n  # closure prep + stage per RK stage


def test_mlp_inference_matches_numpy_restatement():
    from self_b200 import closure as CL
    m = CL.ClosureMLP(seed=11)
    rng = np.random.default_rng(12)
    f = rng.uniform(-1, 1, (4000, 36)).astype(np.float32)
    got = m.infer(torch.from_numpy(f).cuda()).cpu().numpy()
    ref = O.mlp_forward(f.T, *m.unpack())
    assert (ref > 0).any() and (ref < 1).any()
    assert np.abs(got - ref).max() < 1e-5


def test_mlp_closure_tendency_matches_oracle_given_the_same_viscosity():
    """Mode 2: the MLP's activation matches its restatement on the GPU's own
    features, and the viscous path given those viscosities matches the oracle."""
    import self_b200 as S
    from self_b200 import closure as CL
    N = 5
    mod_o, mod, _, q0 = _pair("periodic", N, seed=4)
    mlp = CL.ClosureMLP(seed=5)
    mod.SetClosure(S.CLOSURE_MLP, c=1.0, mlp=mlp)
    got = S.to_host(mod.CalculateTendency()).reshape((N + 1, N + 1, 4, mod.nElem), order="F")
    nu, act, act_ind, (fallbacks, evals) = mod.ClosureState(reset=True)
    assert fallbacks == 0  # untrained ranges are unbounded
    assert 0 < evals < mod.nElem  # the indicator screens out the clearly smooth elements
    _, feat = CL.features(mod.solution, mod.interp)
    ref_act = O.mlp_forward(feat.cpu().numpy().T, *mlp.unpack())
    act_o, _ = O.closure_features(q0, N)
    s_o = _modal_decay_exponent(q0, N)
    screened = s_o < O.default_s0(N) - 1.0 - 1.0  # s < s0 - kappa - 1: a = 0 without the MLP
    ref_act = np.where(screened, 0.0, ref_act)
    assert screened.any() and (~screened).any()
    assert np.abs(act.cpu().numpy() - ref_act).max() < 1e-5
    assert np.abs(act_ind.cpu().numpy() - act_o).max() < 1e-6  # the judge's indicator activations
    mod_o.set_closure(2, c=1.0)
    mod_o.set("avNu", nu.cpu().numpy())
    ref = mod_o.tendency()
    for v in range(4):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL


def test_mlp_fallback_to_indicator_outside_training_range():
    import self_b200 as S
    from self_b200 import closure as CL
    N = 5
    mod_o, mod, _, _ = _pair("periodic", N, seed=6)
    mlp = CL.ClosureMLP(seed=7)
    mlp.fmin[:] = 5.0  # no feature lies in this range: every element falls back
    mlp.fmax[:] = 6.0
    mod.SetClosure(S.CLOSURE_MLP, c=1.0, mlp=mlp)
    mod.CalculateTendency()
    nu, act, act_ind, (fallbacks, evals) = mod.ClosureState(reset=True)
    assert fallbacks == evals > 0  # every element the MLP would evaluate falls back
    np.testing.assert_array_equal(act.cpu().numpy(), act_ind.cpu().numpy())
    mod_o.set_closure(1, c=1.0)
    mod_o.tendency()
    nu_o = mod_o.get("avNu")
    assert np.abs(nu.cpu().numpy() - nu_o).max() <= 1e-6 * nu_o.max()


def test_mlp_training_learns_the_indicator(capsys):
    from self_b200 import closure as CL
    feats, labels = CL.harvest(N_run=7, nx=12, n_problems=3, snapshots=3, steps_between=15, seed=1, N_sample=5)
    assert feats.shape[1] == 36 and feats.shape[0] == labels.shape[0] == 3 * 3 * 144
    assert torch.isfinite(feats).all() and (labels > 0).any()
    mlp = CL.ClosureMLP(seed=2)
    loss = mlp.train(feats, labels, epochs=300, batch=512, lr=3e-3, seed=3)
    pred = mlp.infer(feats)
    mae = float((pred - labels).abs().mean())
    with capsys.disabled():
        print(f"\nclosure MLP: loss {loss[0]:.4f} -> {loss[-1]:.4f}, mean |a_mlp - a_ind| = {mae:.4f} "
              f"over {labels.shape[0]} samples ({int((labels > 0).sum())} active)")
    assert loss[-1] < 0.5 * loss[0]
    assert mae < 0.05


def test_fp32_closure_error_vs_fp64(capsys):
    import self_b200 as S
    N, n = 5, 20
    kw = dict(nx=8, ny=8, periodic=(True, True), perturbation=0.02)
    out = {}
    for form in (S.FP64, S.FP32_BULK):
        interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
        mesh = S.Mesh2D(**kw)
        geo = S.SEMQuad(interp, mesh)
        mod = S.CompressibleIdealGas2D(mesh, geo, form=form)
        q0 = C.shock_state(S.to_host(geo.x), 8, width=0.02)  # x as (2, P, P, 1, nEl)
        mod.SetSolution(q0)
        mod.SetClosure(S.CLOSURE_INDICATOR, c=1.0)
        mod.ForwardStep(n, 1e-4)
        mod.CheckFinite()
        out[form] = mod.solution.clone()
    err = float(torch.linalg.vector_norm(out[S.FP32_BULK] - out[S.FP64]) / torch.linalg.vector_norm(out[S.FP64]))
    with capsys.disabled():
        print(f"\nFP32-bulk closure run: relative L2 error vs FP64 after {n} steps = {err:.3e}")
    assert err < 1e-6  # the bar for the mixed-precision forms


def _full_size_closure_case(S, mesh_o, mesh, N, make_state, steps, form):
    """Indicator-closure tendency and `steps` RK3 steps of a full-size mesh on
    the GPU against the oracle (OpenMP on every host core), 1e-12 relative."""
    import os

    from self_b200 import closure as CL
    O.set_threads(os.cpu_count() or 1)
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    geo = S.SEMQuad(interp, mesh)
    mod = S.CompressibleIdealGas2D(mesh, geo, form=form)
    q0 = make_state(geo.x)
    dt = CL.stable_dt(mod, q0)
    mod.SetSolution(q0)
    mod.SetClosure(S.CLOSURE_INDICATOR, c=1.0)
    mod_o = O.Model(O.CIG, N, mesh_o)
    qh = S.to_host(q0)
    mod_o.set("solution", qh)
    mod_o.set_closure(1, c=1.0)
    ref = mod_o.tendency()
    got = S.to_host(mod.CalculateTendency()).reshape(ref.shape, order="F")
    nu, _, _, _ = mod.ClosureState()
    assert (nu > 0).any()
    for v in range(4):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, ("tendency", v, C.rel_err(got[:, :, v], ref[:, :, v]))
    mod_o.rk3(steps, dt)
    mod.ForwardStep(steps, dt)
    ref = mod_o.get("solution", qh.shape)
    got = S.to_host(mod.solution).reshape(ref.shape, order="F")
    assert np.isfinite(got).all()
    for v in range(4):
        assert C.rel_err(got[:, :, v], ref[:, :, v]) < TOL, ("rk3", v, C.rel_err(got[:, :, v], ref[:, :, v]))


@pytest.mark.parametrize("form", [0, 2])  # production FP64, reference-rounding FP64
def test_c4_full_mesh_indicator_closure_matches_oracle(form):
    """The learned-closure benchmark's mesh at full size: CompressibleIdealGas2D
    periodic 256x256, N = 5, the seeded four-quadrant Riemann problem, with the
    indicator closure: tendency and 10 RK3 steps against the oracle."""
    import self_b200 as S
    from self_b200 import closure as CL
    mk = lambda x: CL.riemann_quadrants(x, np.random.Generator(np.random.PCG64(100)))  # noqa: E731
    _full_size_closure_case(S, O.Mesh(256, 256, periodic=(True, True)),
                            S.Mesh2D(256, 256, periodic=(True, True)), 5, mk, 10, form)


@pytest.mark.parametrize("form", [0, 2])
def test_c5_shaped_mesh_indicator_closure_matches_oracle(form):
    """The large-solve benchmark's shape (periodic, nodes perturbed by 0.02 h,
    N = 7, smooth density wave plus a seeded shock-tube band) on a 256x256
    mesh (a quarter of its 512x512 elements, so that the CPU oracle finishes
    in seconds), indicator closure: tendency and 10 RK3 steps against the
    oracle."""
    import self_b200 as S
    from self_b200 import closure as CL
    mk = lambda x: CL.shock_band(x, np.random.Generator(np.random.PCG64(200)))  # noqa: E731
    _full_size_closure_case(S, O.Mesh(256, 256, periodic=(True, True), amp=0.02),
                            S.Mesh2D(256, 256, periodic=(True, True), perturbation=0.02), 7, mk, 10, form)
