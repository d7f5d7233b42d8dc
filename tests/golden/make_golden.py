"""Generate the golden fixtures under tests/golden/ (run in the build container).

1. ``reference_meshes.json`` -- node coordinates and element corner node ids
   read from the reference's own ISM mesh files
   (etc/mesh/Block2D/Block2D.mesh, etc/mesh/GeophysicalBlock2DMedium/Block2D.mesh
   of the SELF repository).  They pin the structured mesh generator's node
   placement, element ordering and counter-clockwise corner convention.
2. ``oracle_regression.npz`` -- outputs of the CPU oracle on small fixed cases,
   so a later change to the oracle that alters its numbers is caught.

Usage: python tests/golden/make_golden.py <path-to-SELF-checkout>
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)


def read_ism(path):
    """Parse an ISM mesh: 'nNodes nElems nGeo', node lines, then per element
    a corner-id line, a curved-side flag line and a boundary-name line."""
    with open(path) as f:
        lines = [ln.rstrip("\n") for ln in f]
    n_nodes, n_elems, _ = (int(v) for v in lines[0].split())
    nodes = [[float(v) for v in lines[1 + k].split()[:2]] for k in range(n_nodes)]
    elems, bnames = [], []
    k = 1 + n_nodes
    for _ in range(n_elems):
        elems.append([int(v) for v in lines[k].split()])
        bnames.append(lines[k + 2].split())
        k += 3
    return {"nodes": nodes, "elements": elems, "boundary_names": bnames}


def meshes(ref_root):
    out = {}
    for name, rel, box in [
        ("Block2D", "etc/mesh/Block2D/Block2D.mesh", (5, 5, 0.0, 1.0, 0.0, 1.0)),
        ("GeophysicalBlock2DMedium", "etc/mesh/GeophysicalBlock2DMedium/Block2D.mesh",
         (10, 10, -5.0e5, 5.0e5, -5.0e5, 5.0e5)),
    ]:
        d = read_ism(os.path.join(ref_root, rel))
        d["structured"] = box
        d["source"] = rel
        out[name] = d
    return out


def regression():
    from oracle import oracle as O
    rng = np.random.default_rng(1234)
    res = {}
    # CIG on a perturbed periodic 3x3 mesh, N=3, with a smooth random state
    m = O.Mesh(3, 3, periodic=(True, True), amp=0.05)
    mod = O.Model(O.CIG, 3, m)
    x = O.Geometry(3, m).x
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    q = np.zeros((4, 4, 4, 9), order="F")
    rho = 1.0 + 0.1 * np.sin(2 * np.pi * X) * np.cos(2 * np.pi * Y)
    q[:, :, 0], q[:, :, 1], q[:, :, 2] = rho * 0.4, rho * -0.2, rho
    q[:, :, 3] = 1.0 / 0.4 + 0.5 * rho * (0.16 + 0.04)
    mod.set("solution", q)
    res["cig_dSdt"] = mod.tendency()
    mod.rk3(5, 1e-3)
    res["cig_q5"] = mod.get("solution", (4, 4, 4, 9))
    # LSW on a 4x4 reflecting box, N=3
    m = O.Mesh(4, 4, bcid=O.BC_NONORMALFLOW)
    mod = O.Model(O.LSW, 3, m)
    x = O.Geometry(3, m).x
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    q = np.zeros((4, 4, 3, 16), order="F")
    q[:, :, 2] = 0.01 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.01)
    mod.set("H", np.ones((4, 4, 1, 16), order="F"))
    mod.set("solution", q)
    res["lsw_dSdt"] = mod.tendency()
    mod.rk3(5, 1e-3)
    res["lsw_q5"] = mod.get("solution", (4, 4, 3, 16))
    # SW with topography on a 3x3 reflecting box, N=2, one rotated element
    m = O.Mesh(3, 3, bcid=O.BC_NONORMALFLOW, rot=[0, 0, 0, 0, 2, 0, 0, 0, 0])
    mod = O.Model(O.SW, 2, m)
    x = O.Geometry(2, m).x
    X, Y = x[0, :, :, 0, :], x[1, :, :, 0, :]
    h = 0.1 * np.exp(-((X - 0.4) ** 2 + (Y - 0.6) ** 2) / 0.05)
    q = np.zeros((3, 3, 3, 9), order="F")
    q[:, :, 2] = 1.0 + 0.01 * np.exp(-((X - 0.5) ** 2 + (Y - 0.5) ** 2) / 0.02) + rng.uniform(0, 1e-6, X.shape)
    mod.set("topography", h.reshape(3, 3, 1, 9, order="F"))
    mod.set("solution", q)
    res["sw_dSdt"] = mod.tendency()
    mod.rk3(5, 1e-3)
    res["sw_q5"] = mod.get("solution", (3, 3, 3, 9))
    return res


def main():
    if len(sys.argv) < 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the SELF source tree>")
    ref_root = sys.argv[1]
    with open(os.path.join(HERE, "reference_meshes.json"), "w") as f:
        json.dump(meshes(ref_root), f)
    np.savez_compressed(os.path.join(HERE, "oracle_regression.npz"), **regression())


if __name__ == "__main__":
    main()
