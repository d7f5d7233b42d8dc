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
