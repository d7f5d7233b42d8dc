"""Decomposed runs on one GPU: the ranks' handles are stepped stage by stage
from the host with the halo exchange between stages (in-process transport);
the gathered solution equals the single-handle run bit for bit."""
import numpy as np
import pytest
import torch

from tests import cases as C

pytestmark = pytest.mark.gpu


def _build(S, model, mesh, geo, aux, q0):
    cls = {"LSW": S.LinearShallowWater, "SW": S.ShallowWater, "CIG": S.CompressibleIdealGas2D}[model]
    m = cls(mesh, geo)
    if model == "LSW":
        m.SetBathymetry(aux["H"])
        m.SetCoriolis(aux["fCori"])
    elif model == "SW":
        m.SetTopography(aux["topography"])
    m.SetSolution(q0)
    return m


@pytest.mark.parametrize("model,mesh_kind,world", [("CIG", "flipped", 2), ("CIG", "periodic", 3),
                                                   ("LSW", "walls", 2), ("SW", "flipped", 3)])
def test_decomposed_run_equals_single_handle_bitwise(model, mesh_kind, world):
    import self_b200 as S
    from oracle import oracle as O
    from self_b200 import decomp as D
    N, dt, n = 5, 1e-3, 6
    kw = C.mesh_kwargs(mesh_kind)
    gmesh = C.product_mesh(kw)
    interp = S.Lagrange(N, S.GAUSS, N, S.UNIFORM)
    ggeo = S.SEMQuad(interp, gmesh)
    xg = O.Geometry(N, C.oracle_mesh(kw)).x
    aux = C.aux_fields(model, xg, 0)
    q0 = C.initial_state(model, xg, 0)
    ref = _build(S, model, gmesh, ggeo, aux, q0)
    ref.ForwardStep(n, dt)
    ranks = []
    for r in range(world):
        pl = D.HaloPlan(gmesh, world, r)
        lm = pl.local_mesh(gmesh)
        lgeo = S.SEMQuad(interp, lm)
        sl = pl.local_slice()
        laux = {k: np.asfortranarray(v[..., sl]) for k, v in aux.items()}
        ranks.append(D.DecomposedModel(_build(S, model, lm, lgeo, laux, np.asfortranarray(q0[..., sl])), pl))
    assert sum(dm.plan.nHalo for dm in ranks) > 0
    D.LocalTransport().step(ranks, dt, n)
    got = torch.cat([dm.model.solution for dm in ranks])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy(), ref.solution.cpu().numpy())
    assert np.isfinite(got.cpu().numpy()).all()
