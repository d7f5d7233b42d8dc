"""Batched ShallowWater ensembles (uneven instances, per-instance time steps,
one fused handle per degree)."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _small_instances(seed=3):
    from self_b200 import ensemble as E
    return E.make_instances(n=7, seed=seed, nmin=3, nmax=6, degrees=(2, 3, 5))


def test_batched_fp64_equals_unbatched_fp64_bitwise():
    """Batching changes no arithmetic: in the reference-rounding form (the
    kernels' per-element arithmetic is then independent of the kernel the
    autotuner picks) every instance of the batch equals its own run."""
    import self_b200 as S
    from self_b200 import ensemble as E
    inst = _small_instances()
    ens = E.ShallowWaterEnsemble(inst, form=S.FP64_REF, autotune=True)
    ref = E.UnbatchedShallowWater(inst, form=S.FP64_REF)
    ens.ForwardStep(15)
    ref.ForwardStep(15)
    torch.cuda.synchronize()
    for i, (it, model, _) in zip(inst, ref.runs):
        got = ens.solution(i).cpu().numpy()
        assert np.isfinite(got).all()  # assert_array_equal treats NaN == NaN as equal
        np.testing.assert_array_equal(got, model.solution.cpu().numpy())


def test_batched_instance_matches_oracle():
    import self_b200 as S
    from self_b200 import ensemble as E
    inst = _small_instances(seed=5)
    ens = E.ShallowWaterEnsemble(inst, form=S.FP64, autotune=False)
    n = 12
    ens.ForwardStep(n)
    torch.cuda.synchronize()
    for it in inst:
        om = O.Mesh(it.nx, it.ny, bcid=O.BC_NONORMALFLOW)
        mod = O.Model(O.SW, it.N, om)
        x = O.Geometry(it.N, om).x
        X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
        P = it.N + 1
        mod.set("topography", E.topography(it, X, Y).reshape(P, P, 1, -1, order="F"))
        q = np.zeros((P, P, 3, it.nElem), order="F")
        q[:, :, 2] = E.thickness(it, X, Y)
        mod.set("solution", q)
        mod.rk3(n, it.dt)
        ref = mod.get("solution", q.shape)
        got = S.to_host(ens.solution(it)).reshape(q.shape, order="F")
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


def test_fp32_bulk_ensemble_error_vs_fp64(capsys):
    import self_b200 as S
    from self_b200 import ensemble as E
    inst = E.make_instances(n=12, seed=11, nmin=8, nmax=16)
    e64 = E.ShallowWaterEnsemble(inst, form=S.FP64, autotune=False)
    e32 = E.ShallowWaterEnsemble(inst, form=S.FP32_BULK, autotune=True)
    n = 100
    e64.ForwardStep(n)
    e32.ForwardStep(n)
    torch.cuda.synchronize()
    worst = 0.0
    for it in inst:
        a, b = e32.solution(it), e64.solution(it)
        worst = max(worst, float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)))
    with capsys.disabled():
        print(f"\nFP32-bulk ensemble: worst relative L2 error vs FP64 after {n} steps = {worst:.3e}; "
              f"autotune {e32.tuning}")
    assert worst < 1e-6


def _gas_instances(seed=4):
    from self_b200 import ensemble as E
    inst = E.make_gas_instances(n=6, seed=seed, nmin=3, nmax=6, degrees=(5, 7), shock_fraction=0.5)
    assert any(i.smooth for i in inst) and any(not i.smooth for i in inst)
    return inst


def test_gas_ensemble_batched_equals_unbatched_bitwise():
    """CompressibleIdealGas2D instances concatenated per degree advance exactly
    as they do one handle per instance (reference-rounding FP64, no closure)."""
    import self_b200 as S
    from self_b200 import ensemble as E
    inst = _gas_instances()
    ens = E.CompressibleGasEnsemble(inst, form=S.FP64_REF, autotune=True)
    ref = E.UnbatchedGas(inst, form=S.FP64_REF)
    ens.ForwardStep(6)
    ref.ForwardStep(6)
    torch.cuda.synchronize()
    for it, model, _ in ref.runs:
        got = ens.solution(it).cpu().numpy()
        assert np.isfinite(got).all()
        np.testing.assert_array_equal(got, model.solution.cpu().numpy())


def test_gas_ensemble_closure_instance_matches_oracle():
    """A batched instance with the indicator closure (the closure kernels run
    over the concatenated element set) equals the oracle's single-instance
    closure run with the same time step, 1e-12 relative."""
    import self_b200 as S
    from self_b200 import ensemble as E
    from tests import cases as C
    inst = _gas_instances(seed=6)
    ens = E.CompressibleGasEnsemble(inst, form=S.FP64, closure=S.CLOSURE_INDICATOR, autotune=False)
    n = 8
    ens.ForwardStep(n)
    torch.cuda.synchronize()
    for it in inst[:4]:
        om = O.Mesh(it.nx, it.ny, periodic=(True, True), amp=0.02)
        mod = O.Model(O.CIG, it.N, om)
        q0 = ens.handles[it.N]["q0"][it.offset:it.offset + it.nElem]  # the instance's initial state
        mod.set("solution", np.asfortranarray(S.to_host(q0)))
        mod.set_closure(1, c=1.0)
        mod.rk3(n, it.dt)
        ref = mod.get("solution", (it.N + 1, it.N + 1, 4, it.nElem))
        got = S.to_host(ens.solution(it)).reshape(ref.shape, order="F")
        for v in range(4):
            assert C.rel_err(got[:, :, v], ref[:, :, v]) < 1e-12, (it, v, C.rel_err(got[:, :, v], ref[:, :, v]))


def test_gas_ensemble_fp32_learned_error_on_smooth_members(capsys):
    """The batched FP32-bulk + learned-closure form: on smooth members the
    relative L2 error against the plain FP64 run stays within 1e-6."""
    import self_b200 as S
    from self_b200 import closure as CL
    from self_b200 import ensemble as E
    inst = E.make_gas_instances(n=10, seed=12, nmin=6, nmax=12, degrees=(5, 7), shock_fraction=0.3)
    mlps = {5: CL.ClosureMLP(seed=5), 7: CL.ClosureMLP(seed=7)}
    e64 = E.CompressibleGasEnsemble(inst, form=S.FP64, autotune=False)
    e32 = E.CompressibleGasEnsemble(inst, form=S.FP32_BULK, closure=S.CLOSURE_MLP, mlps=mlps, autotune=True)
    n = 50
    e64.ForwardStep(n)
    e32.ForwardStep(n)
    torch.cuda.synchronize()
    worst = 0.0
    for it in inst:
        if it.smooth:  # (the untrained MLPs of this test are not meant to hold the shocks)
            a, b = e32.solution(it), e64.solution(it)
            assert torch.isfinite(a).all()
            worst = max(worst, float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)))
    with capsys.disabled():
        print(f"\nFP32-bulk + learned-closure gas ensemble: worst relative L2 error vs FP64 on smooth members "
              f"after {n} steps = {worst:.3e}")
    assert 0.0 < worst < 1e-6


@pytest.mark.parametrize("form_name", ["FP64", "FP64_REF", "FP32_BULK"])
def test_one_graph_equals_per_handle_replay(form_name):
    """One graph launch per RK step for the whole ensemble (one branch per
    degree) gives the per-handle graph replays' results bit for bit, across
    calls of different lengths, a reset and re-autotuned handles."""
    import self_b200 as S
    from self_b200 import ensemble as E
    form = getattr(S, form_name)
    inst = _small_instances(seed=8)
    one = E.ShallowWaterEnsemble(inst, form=form, autotune=True, one_graph=True)
    per = E.ShallowWaterEnsemble(inst, form=form, autotune=False, one_graph=False)
    for N, h in one.handles.items():  # the same kernel variants in both
        t = one.tuning[N]
        S.lib().selfgpu_model2d_set_launch(per.handles[N]["model"]._h, t["persistent"], t["groups"])
    for n in (1, 4, 3):
        one.ForwardStep(n)
        per.ForwardStep(n)
    torch.cuda.synchronize()
    for it in inst:
        a = one.solution(it).cpu().numpy()
        assert np.isfinite(a).all()
        np.testing.assert_array_equal(a, per.solution(it).cpu().numpy())
    launches = one.launches()
    assert launches == per.launches() and launches > 0
    one.reset()
    per.reset()
    one.ForwardStep(5)
    per.ForwardStep(5)
    torch.cuda.synchronize()
    for it in inst:
        np.testing.assert_array_equal(one.solution(it).cpu().numpy(), per.solution(it).cpu().numpy())
    one.close()


def test_one_graph_gas_closure_equals_per_handle_replay():
    """The closure kernels of every degree are captured into the same
    ensemble graph (indicator closure, production FP64)."""
    import self_b200 as S
    from self_b200 import ensemble as E
    inst = _gas_instances(seed=9)
    one = E.CompressibleGasEnsemble(inst, form=S.FP64, closure=S.CLOSURE_INDICATOR, autotune=False,
                                    one_graph=True)
    per = E.CompressibleGasEnsemble(inst, form=S.FP64, closure=S.CLOSURE_INDICATOR, autotune=False,
                                    one_graph=False)
    one.ForwardStep(7)
    per.ForwardStep(7)
    torch.cuda.synchronize()
    for it in inst:
        a = one.solution(it).cpu().numpy()
        assert np.isfinite(a).all()
        np.testing.assert_array_equal(a, per.solution(it).cpu().numpy())


def test_ensemble_create_rejects_bad_arguments():
    import ctypes

    import self_b200 as S
    from self_b200._lib import lib
    from self_b200 import ensemble as E
    ens = E.ShallowWaterEnsemble(_small_instances(seed=10), form=S.FP64, autotune=False)
    h = next(iter(ens.handles.values()))["model"]._h
    out = ctypes.c_void_p()
    arr = (ctypes.c_void_p * 2)(h, h)
    assert lib().selfgpu_ensemble_create(arr, 2, None, ctypes.byref(out)) != 0  # repeated handle
    assert lib().selfgpu_ensemble_create(arr, 0, None, ctypes.byref(out)) != 0
    assert lib().selfgpu_ensemble_rk3(None, 0.0, 1) != 0
    assert lib().selfgpu_ensemble_destroy(None) == 0
