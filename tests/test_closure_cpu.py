"""CPU pins of the shock closure: modal transform, indicator, features, the
closure MLP restatement and the closure's conservation in the oracle; the
library's host-side modal matrix against the oracle's."""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O
from tests import cases as C


@pytest.mark.parametrize("N", [2, 3, 5, 7])
def test_modal_matrix_maps_legendre_polynomials_to_unit_modes(N):
    """c = T q T^T is exact: the nodal values of Lt_k(x) Lt_l(y) give the unit mode (k, l)."""
    T = O.modal_matrix(N)
    x, _ = O.quadrature(N)
    P = N + 1
    L = np.polynomial.legendre
    for k in range(P):
        for l in range(P):
            lk = L.legval(x, np.eye(P)[k]) * np.sqrt((2 * k + 1) / 2)
            ll = L.legval(x, np.eye(P)[l]) * np.sqrt((2 * l + 1) / 2)
            q = np.outer(lk, ll)  # q[i, j] = Lt_k(x_i) Lt_l(x_j)
            c = T @ q @ T.T
            ref = np.zeros((P, P))
            ref[k, l] = 1.0
            assert np.abs(c - ref).max() < 1e-12


@pytest.mark.parametrize("N", [3, 5, 7])
def test_library_modal_matrix_equals_oracle_bitwise(N):
    from self_b200._lib import lib
    x, w = O.quadrature(N)
    T = np.zeros((N + 1, N + 1), order="F")
    assert lib().selfgpu_modal_matrix(N, x.ctypes.data_as(ctypes.c_void_p), w.ctypes.data_as(ctypes.c_void_p),
                                      T.ctypes.data_as(ctypes.c_void_p)) == 0
    np.testing.assert_array_equal(T, O.modal_matrix(N))


def _state(N, kind, nx=6):
    m = O.Mesh(nx, nx, periodic=(True, True))
    g = O.Geometry(N, m)
    if kind == "smooth":
        return m, C.initial_state("CIG", g.x, 0)
    return m, C.shock_state(g.x, 0)


@pytest.mark.parametrize("N", [5, 7])
def test_indicator_is_off_on_smooth_and_on_across_a_shock(N):
    _, qs = _state(N, "smooth")
    act, feat = O.closure_features(qs, N)
    assert act.max() == 0.0
    _, qk = _state(N, "shock")
    act, feat = O.closure_features(qk, N)
    assert act.max() > 0.3 and (act == 0).any() and ((act > 0) & (act < 1)).any()
    assert np.isfinite(feat).all() and feat.min() >= -1.0 and feat.max() <= 1.0 + 1e-12
    assert feat.shape == (36, qk.shape[3])


def test_constant_state_has_zero_activation():
    N = 5
    m = O.Mesh(3, 3, periodic=(True, True))
    q = np.zeros((6, 6, 4, 9), order="F")
    q[:, :, 2], q[:, :, 3] = 1.0, 2.5
    act, feat = O.closure_features(q, N)
    assert (act == 0).all()
    # a constant has all its energy in mode (0,0): at N = 5 the first shell feature (m = 0) is 1,
    # the five higher shells sit at the floor
    assert np.allclose(feat[0], 1.0) and np.allclose(feat[1:6], -1.0)


def test_bf16_rounding_restatements_agree():
    from self_b200 import closure as CL
    rng = np.random.default_rng(3)
    x = rng.normal(size=1000).astype(np.float32) * 10 ** rng.uniform(-3, 3, 1000).astype(np.float32)
    bits = CL.bf16_bits(x)
    back = (bits.astype(np.uint32) << 16).view(np.float32)
    np.testing.assert_array_equal(back, O.bf16_round(x))
    assert np.abs(back - x).max() <= np.abs(x).max() * 2 ** -8


def test_mlp_forward_clamps_and_matches_a_float64_evaluation():
    from self_b200 import closure as CL
    m = CL.ClosureMLP(seed=4)
    W1, b1, W2, b2, w3, b3 = m.unpack()
    f = np.random.default_rng(5).uniform(-1, 1, (36, 500)).astype(np.float32)
    out = O.mlp_forward(f, W1, b1, W2, b2, w3, b3)
    r = lambda a: O.bf16_round(a).astype(np.float64)  # noqa: E731
    h1 = np.maximum(r(W1) @ f + b1[:, None], 0)
    h2 = np.maximum(r(W2) @ h1 + b2[:, None], 0)
    ref = np.clip(r(w3) @ h2 + b3, 0, 1)
    assert out.min() >= 0 and out.max() <= 1
    assert np.abs(out - ref).max() < 1e-5


@pytest.mark.parametrize("mesh_kind", ["periodic", "walls"])
def test_closure_keeps_the_tendency_conservative(mesh_kind):
    """Sum_ij J w_i w_j dSdt = 0 for mass on periodic meshes, with the viscous
    terms on: the BR1 face flux is the average of both sides' values."""
    N = 5
    kw = C.mesh_kwargs(mesh_kind)
    m = O.Mesh(**kw)
    g = O.Geometry(N, m)
    mod = O.Model(O.CIG, N, m)
    mod.set("solution", C.shock_state(g.x, 1))
    mod.set_closure(1, c=1.0)
    t = mod.tendency()
    nu = mod.get("avNu")
    assert nu.max() > 0
    w = O.quadrature(N)[1]
    wJ = g.J[:, :, 0, :] * w[:, None, None] * w[None, :, None]
    mass = (t[:, :, 2, :] * wJ).sum()
    scale = (np.abs(t[:, :, 2, :]) * wJ).sum()
    # with walls no mass crosses the boundary: the reflected state cancels the
    # inviscid mass flux and physical sides carry no viscous flux
    assert abs(mass) < 1e-12 * scale


def test_closure_off_equals_plain_tendency_and_mode2_with_indicator_nu_equals_mode1():
    N = 5
    m, q = _state(N, "shock", nx=5)
    a = O.Model(O.CIG, N, m)
    a.set("solution", q)
    t0 = a.tendency()
    b = O.Model(O.CIG, N, m)
    b.set("solution", q)
    b.set_closure(1, c=0.7)
    t1 = b.tendency()
    nu = b.get("avNu")
    c = O.Model(O.CIG, N, m)
    c.set("solution", q)
    c.set_closure(2, c=0.7)
    c.set("avNu", nu)
    np.testing.assert_array_equal(c.tendency(), t1)
    b.set_closure(1, c=0.0)  # zero viscosity: the viscous terms add exact zeros
    np.testing.assert_array_equal(b.tendency(), t0)
