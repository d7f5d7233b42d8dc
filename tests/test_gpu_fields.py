"""SELF's field objects (MappedScalar2D / MappedVector2D) on the device: each
type-bound procedure against the oracle's restatement of the same reference
routine, chained in the order SELF's models call them (BoundaryInterp ->
SideExchange -> BassiRebaySides -> GradientBR; ContravariantProjection ->
Divergence), plus Integral against its defining sum."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests import cases as C

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _close(got_t, ref, tol=TOL):
    import self_b200 as S
    got = S.to_host(got_t).reshape(ref.shape, order="F")
    assert C.rel_err(got, ref) < tol, C.rel_err(got, ref)


@pytest.mark.parametrize("N", [3, 6])
@pytest.mark.parametrize("mesh_kind", ["flipped", "periodic"])
def test_mapped_field_procedures_match_oracle(mesh_kind, N):
    import self_b200 as S
    kw = C.mesh_kwargs(mesh_kind)
    om, pm = C.oracle_mesh(kw), C.product_mesh(kw)
    L = S.Lagrange(N)
    Lo = O.Lagrange(N, O.GAUSS, N, O.UNIFORM)
    geo = S.SEMQuad(L, pm)
    go = O.Geometry(N, om)
    nEl, P, nVar = pm.nElem, N + 1, 2
    X, Y = go.x[0, :, :, 0, :], go.x[1, :, :, 0, :]
    f = np.zeros((P, P, nVar, nEl), order="F")
    f[:, :, 0] = np.sin(2 * np.pi * X) * np.cos(np.pi * Y) + 0.3 * X * Y
    f[:, :, 1] = np.exp(-((X - 0.4) ** 2 + (Y - 0.6) ** 2) / 0.1)

    s = S.MappedScalar2D(L, nVar, nEl)
    s.interior.copy_(S.to_device(f))
    s.BoundaryInterp()
    fb = O.scalar_boundary_interp(Lo, f)
    _close(s.boundary, fb)
    s.SideExchange(pm)
    ext = O.side_exchange_scalar(fb, om.sideInfo)
    _close(s.extBoundary, ext)
    s.BassiRebaySides()
    avg = O.bassi_rebay_sides(fb, ext)
    _close(s.avgBoundary, avg)

    g = S.MappedVector2D(L, nVar, nEl)
    s.GradientBR(geo, g)
    gbr = O.gradient_br(Lo, f, avg, go.dsdx, go.J, go.nHat, go.nScale)
    _close(g.interior, gbr)
    gsf = S.MappedVector2D(L, nVar, nEl)
    s.GradientSF(geo, gsf)
    _close(gsf.interior, O.gradient_sf(Lo, f, go.dsdx, go.J))

    # vector procedures on the gradient
    g.BoundaryInterp()
    gb = O.vector_boundary_interp(Lo, gbr)
    _close(g.boundary, gb)
    g.SideExchange(pm)
    _close(g.extBoundary, O.side_exchange_vector(gb, om.sideInfo))
    g.ContravariantProjection(geo)
    gproj = O.contravariant_projection(gbr, go.dsdx)
    _close(g.interior, gproj)
    rng = np.random.default_rng(N)
    bn = np.asfortranarray(rng.standard_normal((P, nVar, 4, nEl)))
    g.boundaryNormal.copy_(S.to_device(bn))
    div = S.MappedScalar2D(L, nVar, nEl)
    g.Divergence(geo, div)
    _close(div.interior, O.jacobian_weight(O.vector_dg_divergence(Lo, gproj, bn), go.J))

    # Integral: variable 4 in the reference; here of each variable of a 4-variable field
    q = S.MappedScalar2D(L, 4, nEl)
    qf = np.zeros((P, P, 4, nEl), order="F")
    qf[:, :, 3] = f[:, :, 0] + 2.0
    qf[:, :, 0] = f[:, :, 1]
    q.interior.copy_(S.to_device(qf))
    w = L.qWeights
    for iVar in (4, 1):
        ref = 0.0
        for e in range(nEl):
            for j in range(P):
                for i in range(P):
                    ref = ref + qf[i, j, iVar - 1, e] * w[i] * w[j] * go.J[i, j, 0, e]
        got = q.Integral(geo, iVar)
        assert abs(got - ref) <= 1e-12 * abs(ref), (iVar, got, ref)
    torch.cuda.synchronize()
