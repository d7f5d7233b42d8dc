"""Multi-rank decomposition on CPU: DomainDecomp / ElemToRank, halo plans,
and the face-trace exchange over gloo with 2 and 3 processes reproducing the
oracle's global SideExchange bit for bit."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _mesh_kwargs():
    return dict(nx=5, ny=4, periodic=(True, True), amp=0.03,
                rot=[0, 1, 2, 3, 2, 0, 3, 1, 1, 3, 0, 2, 3, 2, 1, 0, 2, 1, 0, 3])


def _product_mesh():
    import self_b200 as S
    kw = _mesh_kwargs()
    return S.Mesh2D(kw["nx"], kw["ny"], periodic=kw["periodic"], perturbation=kw["amp"], rotation=kw["rot"])


def test_domain_decomp_and_elem_to_rank_follow_their_definitions():
    from self_b200 import decomp as D
    for nEl in range(1, 61):
        for nd in range(1, min(nEl, 9) + 1):
            off = D.domain_decomp(nEl, nd)
            q, r = divmod(nEl, nd)
            assert list(off) == [d * q + min(d, r) for d in range(nd)] + [nEl]
            for eid in range(1, nEl + 1):
                want = next(d for d in range(nd) if off[d] < eid <= off[d + 1])
                assert D.elem_to_rank(off, eid) == want, (nEl, nd, eid)


@pytest.mark.parametrize("nd", [2, 3, 4])
def test_halo_plans_pair_up_across_ranks(nd):
    from self_b200 import decomp as D
    mesh = _product_mesh()
    si = mesh.sideInfo
    plans = [D.HaloPlan(mesh, nd, r) for r in range(nd)]

    def halo_global(pl):
        """halo slot -> (global element, side) from the local sideInfo."""
        out = {}
        for e in range(pl.nLocal):
            for s in range(4):
                l, g = pl.sideInfo[:, s, e], si[:, s, pl.first + e]
                if l[4] == 0 and l[2] > pl.nLocal:
                    out[l[2] - 1 - pl.nLocal] = (g[2] - 1, g[3] // 10 - 1)
        return out

    for pl in plans:
        assert pl.nHalo == len(halo_global(pl))
        for e in range(pl.nLocal):  # local neighbours keep their (renumbered) ids, flips and sides
            for s in range(4):
                l, g = pl.sideInfo[:, s, e], si[:, s, pl.first + e]
                assert l[3] == g[3] and l[4] == g[4]
                if g[4] == 0 and pl.first <= g[2] - 1 < pl.first + pl.nLocal:
                    assert l[2] == g[2] - pl.first
    for a in plans:
        for p, send, recv in a.peers:
            b = plans[p]
            _, bsend, brecv = next(x for x in b.peers if x[0] == a.rank)
            assert len(send) == len(brecv) and len(recv) == len(bsend)
            hb = halo_global(b)
            for k in range(len(send)):  # what a sends is what b stores for that global side
                s, e = send[k] % 4, send[k] // 4
                hs, he = brecv[k] % 4, brecv[k] // 4 - b.nLocal
                assert hb[he] == (a.first + e, s) and hs == s


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist

    from oracle import oracle as Oo
    from self_b200 import decomp as D
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mesh = _product_mesh()
    N, nVar = 4, 3
    P, nElG = N + 1, mesh.nElem
    L = Oo.Lagrange(N)
    f = np.asfortranarray(np.random.default_rng(1).normal(size=(P, P, nVar, nElG)))
    bnd = Oo.scalar_boundary_interp(L, f)  # (P, nVar, 4, nElG)
    ref = Oo.side_exchange_scalar(bnd, np.asfortranarray(mesh.sideInfo))
    pl = D.HaloPlan(mesh, world, rank)
    nb = 4 * (pl.nLocal + pl.nHalo)
    cache = np.zeros((nb, P * nVar))  # one opaque block per (side, element)
    for e in range(pl.nLocal):
        for s in range(4):
            cache[s + 4 * e] = bnd[:, :, s, pl.first + e].reshape(-1, order="F")
    outgoing = {p: torch.from_numpy(cache[send].copy()).view(torch.uint8).reshape(-1) for p, send, _ in pl.peers}
    sizes = {p: len(recv) * P * nVar * 8 for p, _, recv in pl.peers}
    incoming = D.exchange_buffers(outgoing, sizes)
    for p, _, recv in pl.peers:
        cache[recv] = incoming[p].view(torch.float64).reshape(len(recv), P * nVar).numpy()
    # SideExchange from the local sideInfo and the cache (own or halo blocks, flip applied)
    ok = True
    for e in range(pl.nLocal):
        for s in range(4):
            si = pl.sideInfo[:, s, e]
            if si[4] != 0:
                continue
            e2, s2, flip = si[2] - 1, si[3] // 10 - 1, si[3] % 10
            blk = cache[s2 + 4 * e2].reshape(P, nVar, order="F")
            ext = blk[::-1] if flip else blk
            ok = ok and np.array_equal(ext, ref[:, :, s, pl.first + e])
    out[rank] = (bool(ok), pl.nHalo, len(pl.peers))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_halo_exchange_reproduces_side_exchange(world):
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        ok, nHalo, npeers = res[r]
        assert ok and nHalo > 0 and npeers >= 1
