"""Shared set-ups for the parity tests: the same mesh, geometry, fields and
initial state are built for the oracle and for the CUDA engine."""
import numpy as np

from oracle import oracle as O

MODELS = {"LSW": O.LSW, "SW": O.SW, "CIG": O.CIG}


def rel_err(got, ref):
    got, ref = np.asarray(got), np.asarray(ref)
    scale = np.abs(ref).max()
    return np.abs(got - ref).max() / (scale if scale > 0 else 1.0)


def mesh_kwargs(kind):
    """Named mesh variants: periodic perturbed, walls, walls with rotated
    (flipped-side) elements, prescribed/radiation boundaries."""
    return {
        "periodic": dict(nx=4, ny=3, periodic=(True, True), amp=0.05),
        "walls": dict(nx=3, ny=4, bcid=O.BC_NONORMALFLOW, amp=0.0),
        "flipped": dict(nx=4, ny=3, periodic=(True, False), amp=0.05, bcid=O.BC_NONORMALFLOW,
                        rot=[0, 1, 2, 3, 2, 0, 3, 1, 1, 3, 0, 2]),
        "prescribed": dict(nx=3, ny=3, bcid=O.BC_PRESCRIBED, amp=0.03),
        "radiation": dict(nx=3, ny=3, bcid=O.BC_RADIATION, amp=0.0),
        # edge cases: one element, one column, one row, the smallest periodic
        # mesh (each element meets the other on both sides) with rotated
        # elements, a column periodic across its one-element width (each
        # element is its own east/west neighbour) and one fully periodic element
        "single": dict(nx=1, ny=1, bcid=O.BC_NONORMALFLOW, amp=0.0),
        "ring": dict(nx=1, ny=4, periodic=(True, False), bcid=O.BC_NONORMALFLOW, amp=0.0),
        "torus": dict(nx=1, ny=1, periodic=(True, True), amp=0.0),
        "column": dict(nx=1, ny=5, bcid=O.BC_NONORMALFLOW, amp=0.0),
        "row": dict(nx=7, ny=1, bcid=O.BC_RADIATION, amp=0.0),
        "pair": dict(nx=2, ny=2, periodic=(True, True), amp=0.05, rot=[3, 0, 2, 1]),
    }[kind]


def oracle_mesh(kw):
    return O.Mesh(**kw)


def product_mesh(kw):
    import self_b200 as S
    kw = dict(kw)
    kw["perturbation"] = kw.pop("amp", 0.0)
    kw["rotation"] = kw.pop("rot", None)
    return S.Mesh2D(**kw)


def initial_state(model, x, seed=0):
    """Smooth, seeded initial state on the node coordinates x (2,P,P,1,nEl)."""
    rng = np.random.default_rng(seed)
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    P, nEl = X.shape[0], X.shape[2]
    a, b = rng.uniform(0.5, 1.5, 2)
    if model == "CIG":
        q = np.zeros((P, P, 4, nEl), order="F")
        rho = 1.0 + 0.1 * np.sin(2 * np.pi * a * X) * np.sin(2 * np.pi * b * Y)
        u = 0.5 + 0.05 * np.cos(2 * np.pi * Y)
        v = 0.3 + 0.05 * np.sin(2 * np.pi * X)
        p = 1.0 + 0.05 * np.cos(2 * np.pi * (X + Y))
        q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * u, rho * v, rho
        q[:, :, 3] = p / 0.4 + 0.5 * rho * (u * u + v * v)
        return q
    q = np.zeros((P, P, 3, nEl), order="F")
    bump = np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.05)
    if model == "LSW":
        q[:, :, 0] = 0.01 * np.sin(2 * np.pi * Y) * a
        q[:, :, 1] = 0.01 * np.cos(2 * np.pi * X) * b
        q[:, :, 2] = 0.01 * bump
    else:
        H = 1.0 + 0.01 * bump
        q[:, :, 0] = H * 0.02 * np.sin(2 * np.pi * Y) * a
        q[:, :, 1] = H * 0.02 * np.cos(2 * np.pi * X) * b
        q[:, :, 2] = H
    return q


def aux_fields(model, x, seed=0):
    """Model fields: LSW bathymetry H and Coriolis f, SW topography,
    CIG gravity potential and drag."""
    rng = np.random.default_rng(seed + 1)
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    P, nEl = X.shape[0], X.shape[2]
    if model == "LSW":
        H = (1.0 + 0.1 * np.cos(np.pi * X) * np.cos(np.pi * Y)).reshape(P, P, 1, nEl, order="F")
        f = (rng.uniform(0.5, 1.0) * (1.0 + 0.5 * Y)).reshape(P, P, 1, nEl, order="F")
        return {"H": H, "fCori": f}
    if model == "SW":
        h = (0.1 * np.exp(-((X - 0.3) ** 2 + (Y - 0.6) ** 2) / 0.05)).reshape(P, P, 1, nEl, order="F")
        return {"topography": h}
    phi = (0.5 * Y + 0.1 * X).reshape(P, P, nEl, order="F")
    return {"gravityPotential": phi, "drag": np.full((P, P, nEl), 0.05, order="F")}


def shock_state(x, seed=0, width=0.01):
    """CompressibleIdealGas2D state with an oblique smoothed shock (tanh of the
    given width) and a smooth background: elements across the front activate
    the closure fully, elements near it partly, the rest not at all."""
    rng = np.random.default_rng(seed + 7)
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    P, nEl = X.shape[0], X.shape[2]
    x0, sl = rng.uniform(0.4, 0.6), rng.uniform(0.1, 0.4)
    s = np.tanh((X + sl * Y - x0 - 0.5 * sl) / width)
    rho = 0.8 + 0.3 * s + 0.02 * np.sin(2 * np.pi * Y)
    p = 0.9 + 0.4 * s
    u = 0.2 - 0.1 * s
    v = 0.1 + 0.05 * np.cos(2 * np.pi * X)
    q = np.zeros((P, P, 4, nEl), order="F")
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * u, rho * v, rho
    q[:, :, 3] = p / 0.4 + 0.5 * rho * (u * u + v * v)
    return q
