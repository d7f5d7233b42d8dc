"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its host set-up (quadrature, Lagrange matrices, mesh and
flips, sideInfo validation) agrees bit for bit with the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import self_b200 as S
from oracle import oracle as O
from self_b200 import _lib

HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "selfgpu.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(", src, flags=re.M)
    return sorted(set(n for n in names if n not in ("if", "defined")))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = header_functions()
    assert len(names) >= 50
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_python_signatures_cover_the_header():
    assert set(header_functions()) == set(_lib.exported_symbols())


@pytest.mark.parametrize("N", [1, 2, 3, 4, 5, 6, 7])
@pytest.mark.parametrize("ctrl", [O.GAUSS, O.GAUSS_LOBATTO])
def test_lagrange_matches_oracle_bitwise(N, ctrl):
    if N == 1 and ctrl == O.GAUSS_LOBATTO:
        pytest.skip("degenerate")
    a, b = S.Lagrange(N, ctrl, 2 * N, O.UNIFORM), O.Lagrange(N, ctrl, 2 * N, O.UNIFORM)
    for k in ("controlPoints", "targetPoints", "qWeights", "bWeights", "iMatrix", "dMatrix", "dgMatrix", "bMatrix"):
        np.testing.assert_array_equal(getattr(a, k), getattr(b, k), err_msg=k)


@pytest.mark.parametrize("kw", [
    dict(nx=5, ny=5, bcid=101),
    dict(nx=4, ny=3, periodic=(True, False), amp=0.02, rot=[0, 1, 2, 3] * 3, bcid=102),
    dict(nx=3, ny=4, periodic=(True, True), amp=0.05),
    dict(nx=10, ny=10, x0=-5e5, x1=5e5, y0=-5e5, y1=5e5, bcid=100),
])
def test_mesh_generator_matches_oracle(kw):
    kw = dict(kw)
    o = O.Mesh(**kw)
    kw["perturbation"] = kw.pop("amp", 0.0)
    kw["rotation"] = kw.pop("rot", None)
    m = S.Mesh2D(**kw)
    np.testing.assert_array_equal(m.sideInfo, o.sideInfo)
    np.testing.assert_array_equal(m.nodeCoords, o.nodeCoords)


def _grid_neighbour(nx, ny, periodic, e, s):
    """Unrotated structured grid: the neighbour element and side across local
    side s (0..3 = south, east, north, west) of element e, or None on a
    physical boundary."""
    ix, iy = e % nx, e // nx
    dx, dy = ((0, -1), (1, 0), (0, 1), (-1, 0))[s]
    jx, jy = ix + dx, iy + dy
    if periodic[0]:
        jx %= nx
    if periodic[1]:
        jy %= ny
    if not (0 <= jx < nx and 0 <= jy < ny):
        return None
    return jx + nx * jy, (s + 2) % 4


@pytest.mark.parametrize("nx,ny,periodic", [
    (1, 1, (True, True)), (1, 4, (True, False)), (4, 1, (False, True)), (2, 1, (True, False)),
    (2, 2, (True, True)), (2, 3, (True, True)), (1, 1, (False, False)), (3, 2, (False, True)),
])
def test_narrow_periodic_meshes_connect_grid_neighbours(nx, ny, periodic):
    """Periodic directions one or two elements wide: the two edges of such a
    row share both corner nodes, so sides are matched by their grid edge.
    Every side must meet exactly its grid neighbour (itself across a
    one-element periodic width) with flip 0, and the oracle agrees."""
    m = S.Mesh2D(nx, ny, periodic=periodic, bcid=O.BC_NONORMALFLOW)
    o = O.Mesh(nx, ny, periodic=periodic, bcid=O.BC_NONORMALFLOW)
    np.testing.assert_array_equal(m.sideInfo, o.sideInfo)
    for e in range(nx * ny):
        for s in range(4):
            si = m.sideInfo[:, s, e]
            nb = _grid_neighbour(nx, ny, periodic, e, s)
            if nb is None:
                assert (si[2], si[3], si[4]) == (0, 0, O.BC_NONORMALFLOW), (e, s, si)
            else:
                assert (si[2] - 1, si[3] // 10 - 1, si[3] % 10, si[4]) == (nb[0], nb[1], 0, 0), (e, s, si)
    # global side ids: each interior edge once as +id and once as -id
    ids = m.sideInfo[1][m.sideInfo[4] == 0]
    assert sorted(ids[ids > 0]) == sorted(-ids[ids < 0])


def test_rotation_needs_two_elements_across_a_periodic_direction():
    with pytest.raises(S.SelfGpuError, match="rotated elements"):
        S.Mesh2D(1, 3, periodic=(True, False), rotation=[0, 1, 0])
    S.Mesh2D(1, 3, periodic=(True, False), rotation=[0, 0, 0])
    S.Mesh2D(2, 3, periodic=(True, False), rotation=[0, 1, 2, 3, 0, 1])


def test_side_info_validation_rejects_malformed_records():
    m = S.Mesh2D(3, 3, periodic=(True, True))
    L = _lib.lib()
    ok = np.asfortranarray(m.sideInfo)
    assert L.selfgpu_validate_side_info(ok.ctypes.data_as(ctypes.c_void_p), 9) == 0
    bad = ok.copy(order="F")
    bad[2, 1, 4] = 42  # neighbour id out of range on an interior side
    assert L.selfgpu_validate_side_info(bad.ctypes.data_as(ctypes.c_void_p), 9) == 2
    assert b"invalid neighbour" in L.selfgpu_last_error()
    bad = ok.copy(order="F")
    bad[3, 0, 0] = 57  # neighbour side 5
    assert L.selfgpu_validate_side_info(bad.ctypes.data_as(ctypes.c_void_p), 9) == 2


def test_engine_rejects_bad_arguments_without_a_device():
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.selfgpu_model2d_create(ctypes.byref(h), 9, 7, 10, 0, None) == 1
    assert L.selfgpu_model2d_create(ctypes.byref(h), 3, 12, 10, 0, None) == 1
    assert L.selfgpu_model2d_tendency(None, None) == 1
